/*
 * pim_oracle.h - CPU restatement of the reference CPU_PIM hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA solver:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 * The solver library never links it and never calls it.
 *
 * Every function restates one piece of CPU-PIM/CPU_PIM.cpp (reference repo):
 *   orc_philox4x32_10 / orc_*_word ... random words (replace std::mt19937, see below)
 *   orc_canonical ..................... std::generate_canonical<double,53> (CPU_PIM.cpp:212)
 *   orc_uniform_below ................. std::uniform_int_distribution (CPU_PIM.cpp:147-148)
 *   orc_initial_perms ................. initial shuffle (CPU_PIM.cpp:143-162)
 *   orc_beta_ladder ................... beta ladder (CPU_PIM.cpp:111-119)
 *   orc_force_init .................... force matrix + energy (CPU_PIM.cpp:164-192)
 *   orc_update ........................ one p-dit update (CPU_PIM.cpp:207-287)
 *   orc_update_clique ................. one update of CPU_PIM_tai256c.cpp (:209-337)
 *   orc_replica_sweeps ................ doMegaItera (CPU_PIM.cpp:195-290)
 *   orc_track_exchange ................ best tracking + replica exchange (CPU_PIM.cpp:293-344)
 *   orc_run ........................... threadToRun for all groups in lock step (CPU_PIM.cpp:292-364)
 *   orc_oneshot_* ..................... the one-shot parallel step of GPU-CUPIM (qap.cu:1038-1458),
 *                                       run by orc_run when rule == 1 (parity unpinned: that
 *                                       code needs cuRANDDx and a GPU, neither available here)
 *
 * Random stream.  The reference draws from std::mt19937 seeded by std::random_device, which
 * makes its runs irreproducible.  The solver and this oracle replace the engine by a
 * counter-based Philox4x32-10 stream (Salmon, Moraes, Dror, Shaw, "Parallel Random Numbers:
 * As Easy as 1, 2, 3", SC'11) and consume its 32-bit words exactly where the reference
 * consumes mt19937 words:
 *   - update (group t, replica l, sweep s, location i) takes words 0 and 1 of
 *     Philox(ctr = {i, s, l, t}, key = {seed_lo, seed_hi});
 *   - the initial shuffle takes word k of the shuffle stream from
 *     Philox(ctr = {k / 4, 0, 0, 0xFFFFFFFF}, key)[k % 4].
 * The reference built with an engine shim that returns these words (oracle/ref_prelude.h)
 * follows the same trajectory bit for bit; tests/test_oracle_vs_reference.py checks this.
 *
 * Arithmetic.  Costs, deltas and the force matrix are int64 here (the reference uses int32,
 * which is exact only while no intermediate exceeds 2^31).  Heat-bath weights use x87
 * long double exp2l and double running sums in the reference's order, so the restatement
 * reproduces the reference's picks exactly.
 */
#ifndef PIM_ORACLE_H
#define PIM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The reference's "no best yet" sentinel is INT_MAX (CPU_PIM.cpp:123, :129, :55); the
   int64 restatement keeps the same value so the two agree on every comparison. */
#define ORC_NO_BEST ((int64_t)2147483647)

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
uint32_t orc_sweep_word(uint64_t seed, uint32_t group, uint32_t replica, uint32_t sweep,
                        uint32_t loc, int k);
uint32_t orc_shuffle_word(uint64_t seed, uint64_t k);
double orc_canonical(uint32_t w0, uint32_t w1);
/* uniform_int_distribution<uint32>(0, range-1) on the shuffle stream; *k = next word index. */
uint32_t orc_uniform_below(uint64_t seed, uint64_t *k, uint32_t range);

/* phi[t*n + i] = facility at location i for group t (every replica of a group starts from
   the same permutation, CPU_PIM.cpp:145-161). */
void orc_initial_perms(int n, int T, uint64_t seed, int32_t *phi);
/* beta[l] for l = 0..R-1: beta[R-1] = beta0, beta[l] = beta[l+1] / deltaBeta. */
void orc_beta_ladder(int R, double beta0, double delta_beta, double *beta);

void orc_force_init(int n, const int32_t *D, const int32_t *F, const int32_t *phi,
                    int64_t *I, int64_t *E);

/* One p-dit update of location i.  Returns the picked facility b (== phi[i] for the self
   move), or -1 when no b passes the cumulative test.  dE_out (n entries) is optional. */
int orc_update(int n, const int32_t *D, const int32_t *F, int64_t *I, int32_t *phi,
               int32_t *phiinv, int64_t *E, int64_t *bestE, double beta, int i,
               uint32_t w0, uint32_t w1, int64_t *dE_out);

/* orc_update with the uniform r given directly instead of two engine words. */
int orc_update_r(int n, const int32_t *D, const int32_t *F, int64_t *I, int32_t *phi,
                 int32_t *phiinv, int64_t *E, int64_t *bestE, double beta, int i, double r,
                 int64_t *dE_out);
/* nsweeps sweeps of one replica with the uniforms r[s * n + i] of update (sweep s, location i);
   picks (optional) as orc_replica_sweeps.  Returns the accepted moves. */
int64_t orc_replay_sweeps(int n, const int32_t *D, const int32_t *F, int64_t *I, int32_t *phi,
                          int32_t *phiinv, int64_t *E, int64_t *bestE, double beta, int nsweeps,
                          const double *r, int32_t *picks);

/* nsweeps sweeps of one replica (doMegaItera with NUMITERA = nsweeps).  picks (optional,
   nsweeps*n) records orc_update's return per update.  Returns the number of accepted moves. */
int64_t orc_replica_sweeps(int n, const int32_t *D, const int32_t *F, int64_t *I,
                           int32_t *phi, int32_t *phiinv, int64_t *E, int64_t *bestE,
                           double beta, uint64_t seed, uint32_t group, uint32_t replica,
                           uint32_t sweep0, int nsweeps, int32_t *picks);

/* Best tracking + deterministic exchange for one group at the start of a mega-iteration
   (CPU_PIM.cpp:295-344).  order has cap entries (the reference's MAXNUMREPLICAS); entries
   past R keep their value between calls.  *single_best is the cross-group best.
   Returns 1 when the group best improved (foundBetter). */
int orc_track_exchange(int R, int cap, const int64_t *E, const int64_t *bestE, double *beta,
                       int32_t *order, int32_t *time_since_swap, int64_t *thread_best,
                       int64_t *single_best);

/* Whole-run state for T groups x R replicas (arrays indexed [t*R + l] / [(t*R + l)*n + i]). */
typedef struct orc_run_state {
    int n, T, R, cap, numitera;
    uint64_t seed;
    int64_t *I;          /* T*R*n*n */
    int32_t *phi;        /* T*R*n */
    int32_t *phiinv;     /* T*R*n */
    int64_t *E;          /* T*R */
    int64_t *bestE;      /* T*R */
    double *beta;        /* T*R, by replica slot */
    int32_t *order;      /* T*cap */
    int32_t *time_since_swap; /* T */
    int64_t *thread_best;     /* T */
    int64_t single_best;
    int64_t megaiters_done;   /* mega-iterations completed (exchange + sweeps) */
    int64_t accepts;
    int64_t target_megaiter;  /* first mega-iteration whose tracking saw single_best <= goal, or -1 */
    int32_t active;           /* 0: orc_update; A > 0: orc_update_clique with A active facilities */
    int32_t rule;             /* 0: the sequential p-dit sweeps; 1: one-shot steps (orc_oneshot_step) */
} orc_run_state;

/* ---- the one-shot parallel update of GPU-CUPIM (perl-gpu/src/lib/qap/qap.cu:1038-1458) ----
   One step of a replica: every location i proposes a partner j against the same snapshot
   (heat-bath weights over all n partners in binary32, no cutoff, summed in the reference's
   warp order), collisions go to the proposal with the larger delta (then the lower i), the
   surviving swaps (disjoint pairs) are applied together, and the energy is recomputed from the
   updated force matrix.  The reference's cuRANDDx uniforms are replaced by word 0 of the
   update's Philox block (orc_sweep_word with sweep = step).  Returns the swaps applied;
   targets (optional, n entries) receives every location's proposal. */
float orc_exp2f_neg(float x);
float orc_oneshot_uniform(uint32_t w0);
/* The thresholds of one step of `count` replicas, replica k being replica k % R of group k / R:
   out[k][i] = orc_oneshot_uniform(word 0 of (group, replica, step, location i)). */
void orc_oneshot_uniforms(uint64_t seed, int count, int R, uint32_t step, int n, float *out);
int orc_oneshot_pick(int n, const int64_t *d, float beta_f, float u, int64_t *delta_out);
int orc_oneshot_step(int n, const int32_t *D, const int32_t *F, int64_t *I, int32_t *phi,
                     int32_t *phiinv, int64_t *E, int64_t *bestE, double beta, uint64_t seed,
                     uint32_t group, uint32_t replica, uint32_t step, int32_t *targets);

/* The clique-flow update of CPU-PIM/CPU_PIM_tai256c.cpp (doMegaIteraTai, :209-337), with the
   reference's hard-wired 92 active facilities and n = 256 made parameters: facilities
   0..act-1 form a clique of unit flows, the others have no flow at all (so every swap between
   two of them leaves the energy and the force matrix unchanged), and D, F have zero diagonals.
   A location holding an inactive facility weighs the active facilities one by one and all
   inactive ones as one lumped candidate (weight (n - act) * exp2(beta * dE(act)), never cut
   off, :253-266); when the lumped candidate is drawn, the facility to swap with is
   act + uniform_int(n - act) (:324-336) on the words of orc_lumped_word.  Returns the facility
   swapped in (phi[i] for no move) or -1. */
int orc_update_clique(int n, int act, const int32_t *D, const int32_t *F, int64_t *I,
                      int32_t *phi, int32_t *phiinv, int64_t *E, int64_t *bestE, double beta,
                      int i, uint32_t w0, uint32_t w1, uint64_t seed, uint32_t group,
                      uint32_t replica, uint32_t sweep);

/* Words of the lumped draw of update (group, replica, sweep, loc): words 2 and 3 of the
   update's Philox block, then blocks with counter word 3 = group + 0x10000 * m, m >= 1. */
uint32_t orc_lumped_word(uint64_t seed, uint32_t group, uint32_t replica, uint32_t sweep,
                         uint32_t loc, uint32_t k);

/* setup(): ladder, shuffle, force matrices, energies (CPU_PIM.cpp:109-193).  The caller
   allocates every array of st and fills n, T, R, cap, numitera, seed. */
void orc_setup(orc_run_state *st, const int32_t *D, const int32_t *F, double beta0,
               double delta_beta);
/* megaiters mega-iterations of threadToRun for all groups, lock step: every group does its
   tracking + exchange, then the goal test (stop when single_best <= goal), then every group
   sweeps.  Returns 1 when the goal stopped the run. */
int orc_run(orc_run_state *st, const int32_t *D, const int32_t *F, int64_t megaiters,
            int64_t goal);

#ifdef __cplusplus
}
#endif
#endif
