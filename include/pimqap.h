/*
 * pimqap.h - C ABI of the B200 parallel-tempering p-dit QAP solver.
 *
 * The solver is a drop-in for the reference's CPU_PIM path (CPU-PIM/CPU_PIM.cpp): the same
 * instance file, the same replica / temperature / sweep parameters and the same outputs.
 * The reference has no library interface: its path is the CLI main() over global arrays
 * with compile-time capacities.  Each entry point below names the reference function or
 * block it replaces.
 *
 * Conventions
 *   - Every function returns a pimqap_status (0 = OK).  No exception crosses the ABI.
 *     pimqap_last_error() gives the message of the calling thread's last failure.
 *   - All pointers are caller-owned host memory unless stated otherwise; the solver copies
 *     what it needs.  Device memory is owned by the solver / server handles.  A destroyed
 *     solver handle's device block of up to 256 MiB is kept (one per GPU, until the process
 *     exits) for the next handle on that GPU, so repeated solves skip cudaMalloc / cudaFree.
 *   - A solver handle is used by one host thread at a time.  A server handle is locked
 *     internally and may be used from several threads.
 *   - Energies and costs are exact int64.  The force matrix is int32 when a bound computed
 *     from the instance proves every value fits, else int64 (or as forced by params).
 *   - Random words come from a counter-based Philox4x32-10 stream keyed by params.seed, so a
 *     run is a pure function of (instance, params) and does not depend on what else runs on
 *     the GPU.
 */
#ifndef PIMQAP_H
#define PIMQAP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PIMQAP_MAX_N 256          /* reference: MAXN = 160 (CPU_PIM.cpp:16) */
#define PIMQAP_MAX_REPLICAS 64    /* reference: MAXNUMREPLICAS = 10 (CPU_PIM.cpp:23) */
#define PIMQAP_MAX_GROUPS 1024    /* reference: MAXNUMTHREADS = 20 (CPU_PIM.cpp:26) */
/* "No best energy yet": the reference's INT_MAX sentinel (CPU_PIM.cpp:123, :129). */
#define PIMQAP_NO_BEST ((int64_t)2147483647)

typedef enum pimqap_status {
    PIMQAP_OK = 0,
    PIMQAP_ERR_ARG = 1,        /* invalid argument (n, replicas, groups, beta, ...) */
    PIMQAP_ERR_IO = 2,         /* instance file missing or malformed */
    PIMQAP_ERR_CUDA = 3,       /* CUDA runtime failure (message has the CUDA error) */
    PIMQAP_ERR_NO_DEVICE = 4,  /* no sm_100 device, or the kernels are not loadable */
    PIMQAP_ERR_RANGE = 5,      /* instance values overflow the int64 bound */
    PIMQAP_ERR_DEVICE = 6,     /* a device-side check failed (error word set) */
    PIMQAP_ERR_BUSY = 7,       /* server queue full / memory budget exhausted */
    PIMQAP_ERR_NOT_READY = 8,  /* server ticket not finished yet */
} pimqap_status;

/* One QAP instance.  flow is F (n x n, facility x facility) and dist is D (n x n, location
   x location), both row-major int32, in the order the reference's file lists them
   (CPU_PIM.cpp:94-103). */
typedef struct pimqap_instance {
    int32_t n;
    const int32_t *flow;
    const int32_t *dist;
} pimqap_instance;

/* Solve parameters; the CLI flag of the reference is given for each field
   (CPU_PIM.cpp:478-610). */
typedef struct pimqap_params {
    int32_t replicas;            /* -r  replicas per group (NUMREPLICAS) */
    int32_t groups;              /* -t  independent parallel-tempering groups (NUMTHREADS) */
    int32_t sweeps_per_exchange; /* -i  sweeps between replica exchanges (NUMITERA, default 4) */
    int32_t rank_slots;          /* the reference's compiled MAXNUMREPLICAS, which places the
                                    forced extreme swap (CPU_PIM.cpp:340); 0 = max(replicas, 10) */
    int64_t max_megaiters;       /* -w  mega-iterations (exchange + sweeps_per_exchange sweeps) */
    double beta_max;             /* -b  largest beta in natural units (stored x 1/ln2, :528) */
    double beta_ratio;           /* -m  divisive step between adjacent betas (deltaBeta) */
    int64_t goal;                /* -g  stop once the best energy is <= goal */
    double timeout_s;            /* -s  stop after this many seconds (0 = none) */
    uint64_t seed;               /* Philox key */
    int32_t force_bits;          /* 0 = choose from the instance bound, 32 or 64 = force */
    int32_t device;              /* CUDA device ordinal */
    int32_t megaiters_per_launch;/* mega-iterations per CUDA-graph launch (0 = automatic) */
    int32_t threads_per_block;   /* 0 = automatic, else 64, 128 or 256 (also 32 for n <= 128
                                    with the sequential rule, 512 with the one-shot rule): the
                                    threads of one replica's CTA */
    int32_t cluster_size;        /* CTAs per replica: 0 = smallest that fits, else 1, 2 or 4 */
    int32_t beta_internal;       /* nonzero: beta_max is already in the reference's internal
                                    (log2) units, as automatic mode sets beta0 = 2^k (:397) */
    int32_t auto_beta;           /* nonzero: choose beta_max / beta_ratio by the reference's
                                    automatic mode before solving (no -b flag, :645-658) */
    double auto_lower;           /* -al lowerBetaProportion (default 0.1, :33) */
    double auto_higher;          /* -ah higherBetaProportion (default 0.9, :34) */
    int64_t goal_print;          /* -G  record a replica whose best falls below this during a
                                    sweep, with its permutation (goalPrint, :271-282); acts only
                                    when > 0, as in the reference.  Needs event_capacity > 0 */
    int32_t event_capacity;      /* progress events kept per run call (0 = no event log); see
                                    pimqap_solver_events */
    int32_t event_perm_capacity; /* goal_print permutations kept per run call (0 = 256) */
    int32_t compact_instance;    /* 0 = automatic: a symmetric instance with 0/1 flows and
                                    int16 distances keeps D and F in shared memory beside the
                                    force rows (same results); 1 = never */
    int32_t active_facilities;   /* > 0: the moves of the reference's tai256c program
                                    (CPU-PIM/CPU_PIM_tai256c.cpp, which hard-wires 92 of 256):
                                    facilities 0..A-1 must form a clique of unit flows and the
                                    others carry none; a location holding an inactive facility
                                    weighs the actives and all inactives as one lumped move.
                                    pimqap_solve / solver handles only; no goal_print events */
    int32_t update_rule;         /* PIMQAP_RULE_SEQUENTIAL (0): CPU_PIM's sweeps, one location
                                    after another; PIMQAP_RULE_ONE_SHOT (1): the one-shot
                                    parallel step of GPU-CUPIM (perl-gpu/src/lib/qap/qap.cu:
                                    1038-1458), which every location of a replica proposes a
                                    partner in against the same snapshot, collisions go to the
                                    larger delta and the surviving swaps apply together; a
                                    "sweep" is then one such step.  pimqap_solve / solver
                                    handles only */
    int32_t replica_pairing;     /* binary-flow instances (symmetric 0/1 flows, int16 distances):
                                    0 = automatic (one replica per CTA set: measured faster),
                                    1 = one replica per CTA (or cluster), 2 = two replicas of
                                    the instance per CTA (or cluster), each on half of its warps
                                    over one shared copy of the instance, so their update chains
                                    interleave.  Same results either way.  pimqap_solve / solver
                                    handles only */
    int32_t launch_mode;         /* 0 = automatic (= 1, measured as fast or faster);
                                    1 = a launch per mega-iteration (CUDA graphs of
                                    megaiters_per_launch); 2 = one persistent launch per run
                                    call with a device-side barrier between mega-iterations
                                    (every replica resident at once, no event log; rejected
                                    otherwise).  Same results either way.  pimqap_solve /
                                    solver handles only */
    int32_t sweep_pipeline;      /* binary-flow instances: 0 = automatic (off), 1 = off,
                                    2 = compute each update's deltas while the previous update
                                    picks (half of a CTA's warps pick, half compute the next
                                    deltas against the state before the pick's swap and then
                                    correct them for it).  Same results either way; with
                                    launch_mode 0 / 1, one replica per CTA set, no clique moves */
    int32_t tensor_update;       /* the force update on the tensor cores.  One-shot rule: 0 =
                                    automatic (tcgen05 where exact and it fits, else mma.sync
                                    where exact, else the integer CUDA cores), 1 = integer CUDA
                                    cores, 2 = the legacy tensor-core path (mma.sync m16n8k16),
                                    3 = tcgen05 (fp16 factors in shared memory, the step's sums
                                    in tensor memory; at most 128 rows per CTA and n <= 256);
                                    2 and 3 need factors fp16 holds exactly (2 dD or dD, and
                                    dF, at most 2048 in magnitude) and n |dD| |dF| < 2^24.
                                    Sequential rule (the binary-flow kernel's rewrite of its
                                    rows every 16 accepted swaps): 0 = automatic (tcgen05 where
                                    the distance range is at most 1024, n <= 256 and the
                                    threads per block a multiple of 128, else binary32 FMAs on
                                    the CUDA cores), 1 = the CUDA cores, 3 = tcgen05 (rejected
                                    where it does not apply; the paired and pipelined epochs
                                    keep the CUDA cores), 2 = rejected.  The same integer
                                    results in every form */
    int32_t oneshot_weights;     /* the one-shot rule's binary32 2^x: 0 = CUDA's exp2f, the
                                    function GPU-CUPIM's proposals call (qap.cu:1083-1086),
                                    written as the reference writes it, so a step takes the
                                    reference kernels' decisions; 1 = this library's own 2^x
                                    (Cody-Waite reduction, degree-7 polynomial, under 1 ulp),
                                    which the CPU oracle restates bit for bit.  One-shot rule
                                    only */
} pimqap_params;

#define PIMQAP_RULE_SEQUENTIAL 0
#define PIMQAP_RULE_ONE_SHOT 1

/* Fills p with the reference's defaults: 10 replicas, 20 groups, 4 sweeps per exchange,
   beta_ratio 1.2 (CPU_PIM.cpp:19-31), no goal, no timeout, seed 1, automatic shapes. */
void pimqap_default_params(pimqap_params *p);

typedef struct pimqap_result {
    int64_t best_energy;        /* best energy of any visited state (PIMQAP_NO_BEST if none) */
    int32_t *best_perm;         /* caller-provided, n entries (may be NULL): facility at each
                                   location for best_energy */
    int64_t target_megaiter;    /* mega-iteration whose tracking first saw best <= goal, or -1 */
    double time_to_target_ms;   /* device time from the first sweep to that tracking, or -1 */
    int64_t megaiters_done;     /* mega-iterations completed */
    int64_t updates;            /* p-dit updates over all replicas */
    int64_t accepts;            /* accepted swaps over all replicas */
    double device_ms;           /* device time of the sweep launches */
    double wall_ms;             /* host wall time of the whole call */
    int32_t force_bits;         /* 32 or 64: the force-matrix width used */
    int32_t cluster_size;       /* CTAs per replica (1, 2 or 4) */
    int32_t stopped_by;         /* 0 = max_megaiters, 1 = goal, 2 = timeout */
    int32_t launches;           /* kernel launches of the sweeps (solver path): one per
                                   mega-iteration, or one per run call when persistent */
    int64_t h2d_bytes;          /* host-to-device bytes copied by the solver so far */
    int64_t d2h_bytes;          /* device-to-host bytes copied by the solver so far */
    int64_t *final_energies;    /* caller-provided, groups * replicas entries (may be NULL):
                                   currentE of every replica at the end (CPU_PIM.cpp:54) */
    double beta_max_used;       /* beta0 of the run in internal units (after automatic mode) */
    double beta_ratio_used;     /* deltaBeta of the run */
    double admit_ms;            /* serving: submit -> admitted to the device (host clock) */
    double latency_ms;          /* serving: submit -> result available (host clock) */
    int64_t sweeps;             /* replica-sweeps over all replicas (updates / n) */
    int64_t proposals;          /* swap proposals, n (n - 1) / 2 per replica-sweep */
} pimqap_result;

/* ---------------------------------------------------------------- instance I/O */

/* Reads a reference instance file (replaces readProblem, CPU_PIM.cpp:79-107): n, then F,
   then D, whitespace separated.  Call with flow = dist = NULL to get n; then with arrays
   of n*n entries.  n > max_n is rejected like the reference's MAXN check (:88-92). */
pimqap_status pimqap_read_problem(const char *path, int32_t max_n, int32_t *n,
                                  int32_t *flow, int32_t *dist);

/* The same reader (readProblem, CPU_PIM.cpp:79-107) into arrays it allocates: inst->flow and
   inst->dist hold n*n entries each until pimqap_free_instance releases them. */
pimqap_status pimqap_load_file(const char *path, pimqap_instance *inst);
void pimqap_free_instance(pimqap_instance *inst);

/* ---------------------------------------------------------------- one-shot solve */

/* The whole CPU_PIM run with fixed beta parameters (replaces setup() + the threadToRun
   loop, CPU_PIM.cpp:109-364 and :636-684): uploads the instance, builds the replicas,
   runs max_megaiters mega-iterations (or until goal / timeout) on the GPU and returns the
   best energy and permutation. */
pimqap_status pimqap_solve(const pimqap_instance *inst, const pimqap_params *params,
                           pimqap_result *result);

/* One-shot solve that allocates nothing (no counterpart in the reference, whose CPU solver
   has no device memory).  For callers that must not call cudaMalloc while they solve: a
   program whose device memory is all claimed by another allocator (a framework's caching
   allocator, a service that admits work against memory reserved up front), or code that may
   not take the allocator's locks or latency.  Same inputs, outputs and results as
   pimqap_solve, but every device buffer lives in one file-scope device array of
   PIMQAP_STATIC_SCRATCH_BYTES that each GPU holds from library load until exit; a solve that
   needs more is rejected with PIMQAP_ERR_ARG.  The first call on a device looks the array's
   address up (make it before any stream capture).  Calls share the array: this library
   serialises its own calls per device, and calls that overlap on one GPU from elsewhere race.
   Work runs on the legacy default stream; no stream, event or graph is created, so
   result->device_ms is the host wall time of the launch loop here, not an event-timed
   device figure like pimqap_solve's. */
#define PIMQAP_STATIC_SCRATCH_BYTES ((size_t)8 << 20)
pimqap_status pimqap_solve_static(const pimqap_instance *inst, const pimqap_params *params,
                                  pimqap_result *result);

/* ---------------------------------------------------------------- solver handle */

typedef struct pimqap_solver pimqap_solver;

/* setup() on the device (CPU_PIM.cpp:109-193): beta ladder, initial shuffle, force
   matrices, energies, and the tracking/exchange step of mega-iteration 0. */
pimqap_status pimqap_solver_create(const pimqap_instance *inst, const pimqap_params *params,
                                   pimqap_solver **out);

/* Runs megaiters more mega-iterations (threadToRun's loop body, CPU_PIM.cpp:293-362):
   sweeps_per_exchange sweeps of every replica (doMegaItera, :195-290), then each group's
   best tracking and replica exchange.  Stops early when the goal is reached.  If device_ms
   is not NULL it receives the device time measured with CUDA events on the solver's stream.
   Returns after the work completes. */
pimqap_status pimqap_solver_run(pimqap_solver *s, int64_t megaiters, double *device_ms);

/* Best energy, permutation and counters so far. */
pimqap_status pimqap_solver_result(pimqap_solver *s, pimqap_result *result);

/* Full state of replica l of group t, for parity checks against the reference's globals
   facilityOfLocation / locationOfFacility / I / currentE / bestE / beta (CPU_PIM.cpp:44-62).
   I (n*n, row-major) is returned widened to int64.  Any output pointer may be NULL. */
pimqap_status pimqap_solver_replica(pimqap_solver *s, int32_t t, int32_t l, int32_t *phi,
                                    int64_t *force, int64_t *energy, int64_t *best_energy,
                                    double *beta);

/* Exchange state of group t: indexOfBetaOrder (rank_slots entries), timeSinceSwap and
   threadBestE (CPU_PIM.cpp:44, :52, :69). */
pimqap_status pimqap_solver_group(pimqap_solver *s, int32_t t, int32_t *order,
                                  int32_t *time_since_swap, int64_t *group_best);

/* A progress event: what the reference prints while it runs, recorded on the device with
   the time it happened.  Recorded only when params.event_capacity > 0. */
#define PIMQAP_EVENT_GROUP_BEST 0 /* tracking of mega-iteration `megaiter` found replica
                                     `replica` below group `group`'s best (threadBestE); one
                                     event per lowering, in the reference's replica order
                                     (CPU_PIM.cpp:297-314).  "Best Energy Found" lines are the
                                     events that also lower the best over all groups (:303-311)
                                     and sweep<t>.txt holds the last event of each (m, t) (:317-321) */
#define PIMQAP_EVENT_GOAL_PRINT 1 /* a sweep of mega-iteration `megaiter` lowered the replica's
                                     best below params.goal_print (:271-282) */
typedef struct pimqap_event {
    int64_t megaiter;
    int64_t energy;
    double time_ms;             /* device time since setup (solver) or the batch start */
    int32_t kind;               /* PIMQAP_EVENT_* */
    int32_t group;
    int32_t replica;
    int32_t perm_index;         /* GOAL_PRINT: argument of pimqap_solver_event_perm, -1 when the
                                   permutation store of that run call was full */
    int32_t trial;              /* automatic mode: trial index (beta step * 5 + trial); else 0 */
    int32_t pad;
} pimqap_event;

/* Events recorded so far, in the reference's order (mega-iteration, then tracking before the
   sweeps, then group, then replica): copies events [first, first + capacity) into `events`
   and sets *count to the number copied.  *total (may be NULL) receives the number recorded;
   *dropped (may be NULL) the number lost because a run call recorded more than
   params.event_capacity. */
pimqap_status pimqap_solver_events(pimqap_solver *s, int64_t first, int32_t capacity,
                                   pimqap_event *events, int32_t *count, int64_t *total,
                                   int64_t *dropped);

/* The permutation (n entries) of a GOAL_PRINT event. */
pimqap_status pimqap_solver_event_perm(pimqap_solver *s, int32_t perm_index, int32_t *perm);

void pimqap_solver_destroy(pimqap_solver *s);

/* No counterpart in the reference (its memory is static arrays).  Frees the device blocks that
   destroyed solver handles left for reuse (one per GPU, up to 256 MiB each).  Call it before
   cudaDeviceReset or before handing the memory to other code; the next solve allocates anew.
   Returns the first cudaFree error as PIMQAP_ERR_CUDA; with nothing kept it makes no CUDA
   call. */
pimqap_status pimqap_release_kept_memory(void);

/* Parity tool: nsweeps sweeps of ONE replica (doMegaItera, CPU_PIM.cpp:195-290, with NUMITERA
   sweeps and no exchange partner) from the caller's permutation phi_in (facility at each
   location), at beta = params->beta_max (natural units unless params->beta_internal), with the
   uniform r of every update given by the caller (r[s * n + i] for sweep s, location i, each in
   [0, 1); the reference draws it with generate_canonical, :212) instead of the Philox stream.
   The force matrix is set up from phi_in on the device (:164-192).  Outputs (any may be NULL):
   the final permutation (n), force matrix (n*n, widened to int64), energy, best energy and
   accepted moves.  Force width and launch shape follow params; the sequential rule only. */
pimqap_status pimqap_sweep_replay(const pimqap_instance *inst, const pimqap_params *params,
                                  const int32_t *phi_in, int32_t nsweeps, const double *r,
                                  int32_t *phi_out, int64_t *force, int64_t *energy,
                                  int64_t *best_energy, int64_t *accepts);

/* ---------------------------------------------------------------- batched solve */

/* Many independent instances of uneven n, each with its own replica set and parameters,
   in one persistent launch (no reference counterpart: the reference solves one instance
   per process).  results[k].best_perm must hold insts[k].n entries or be NULL.
   Each result equals what pimqap_solve returns for that instance alone. */
pimqap_status pimqap_batch_solve(const pimqap_instance *insts, const pimqap_params *params,
                                 int32_t count, pimqap_result *results);

/* The same batch without blocking: pimqap_batch_submit copies the instances and parameters and
   returns at once; the batch runs on a host thread of its own.  The caller's results array
   (with its best_perm / final_energies buffers) is written when the batch finishes and must
   stay alive until pimqap_batch_poll returns PIMQAP_OK (PIMQAP_ERR_NOT_READY before) or
   pimqap_batch_wait (up to timeout_s seconds, < 0 = no limit) does; then release the handle. */
typedef struct pimqap_batch pimqap_batch;
pimqap_status pimqap_batch_submit(const pimqap_instance *insts, const pimqap_params *params,
                                  int32_t count, pimqap_result *results, pimqap_batch **out);
pimqap_status pimqap_batch_poll(pimqap_batch *b);
pimqap_status pimqap_batch_wait(pimqap_batch *b, double timeout_s);
void pimqap_batch_release(pimqap_batch *b);

/* The autotuner of the batched solve (no reference counterpart): a batch's instances fall into
   classes (force width x CTAs per replica x band of n), each run by one persistent launch.  For
   each class shape it has not seen yet in this process, the tuner times one mega-iteration of
   the class's instances under every candidate worker shape (threads per replica 32-256 x
   replicas per CTA) and keeps the fastest; pimqap_batch_solve then uses the cached choice.
   Shapes never change results.  pimqap_batch_tune runs the tuner on a batch without solving it
   and reports each class; with PIMQAP_AUTOTUNE=0 in the environment the batch keeps the fixed
   rules' shapes (the report then has tried = 0). */
typedef struct pimqap_class_tuning {
    int32_t force_bits, cluster_size, band, n_max, members;
    int32_t threads, workers, grid;              /* the shape in use: threads per replica,
                                                    replicas per CTA, CTAs of the launch */
    int32_t fixed_threads, fixed_workers;        /* the fixed rules' shape */
    int32_t tried;                               /* shapes timed when the class was tuned */
    int32_t pad;
    double fixed_ms, tuned_ms;                   /* device time of one mega-iteration of the
                                                    class's instances under each shape */
} pimqap_class_tuning;
pimqap_status pimqap_batch_tune(const pimqap_instance *insts, const pimqap_params *params,
                                int32_t count, pimqap_class_tuning *classes, int32_t capacity,
                                int32_t *class_count);

/* ---------------------------------------------------------------- serving */

/* Continuous-batching solve service (no reference counterpart).  Persistent launches stay
   resident on the device, one per class of replica shape; a server thread admits submitted
   requests in arrival order as instance slots and device memory (the budget) free up, and
   the running launches pick them up between epochs, so new work overlaps work in flight.
   Each result equals what pimqap_solve returns for that request alone.  The handle is
   internally locked; submit / poll / wait may be called from several threads. */
typedef struct pimqap_server pimqap_server;

typedef struct pimqap_server_config {
    int32_t device;
    int64_t memory_budget_bytes;   /* device memory for admitted requests (0 = half of free) */
    int32_t slots_per_class;       /* requests resident at once per class (0 = 256) */
    double heartbeat_timeout_s;    /* device workers stop if the server thread stalls this long
                                      (0 = 10 s) */
    /* Representative requests for the autotuner, which sizes the classes and their share of
       the SMs from them (NULL / 0 = a built-in mix of n = 32..256, int32 and int64). */
    const pimqap_instance *sample;
    const pimqap_params *sample_params;
    int32_t sample_count;
} pimqap_server_config;

typedef struct pimqap_server_stats {
    int64_t submitted, admitted, completed, pending;
    int64_t memory_in_use, memory_budget;
    int32_t classes;
    int32_t error_word;            /* device error bits of any class launch (0 = healthy) */
} pimqap_server_stats;

pimqap_status pimqap_server_create(const pimqap_server_config *config, pimqap_server **out);
/* Queues a request (the instance is copied; the caller may free it on return).  *ticket
   identifies it.  PIMQAP_ERR_BUSY when it can never fit the memory budget or no class
   fits its shape. */
pimqap_status pimqap_server_submit(pimqap_server *s, const pimqap_instance *inst,
                                   const pimqap_params *params, int64_t *ticket);
/* PIMQAP_ERR_NOT_READY while the request is pending or running; then fills result (and its
   best_perm / final_energies arrays when given) and forgets the ticket. */
pimqap_status pimqap_server_poll(pimqap_server *s, int64_t ticket, pimqap_result *result);
/* Like poll, waiting up to timeout_s (< 0: no limit). */
pimqap_status pimqap_server_wait(pimqap_server *s, int64_t ticket, double timeout_s,
                                 pimqap_result *result);
pimqap_status pimqap_server_stats_get(pimqap_server *s, pimqap_server_stats *stats);
/* Stops the launches and frees the device memory.  Requests not finished yet are abandoned
   (their tickets become invalid): wait for the ones whose results are needed first. */
void pimqap_server_destroy(pimqap_server *s);

/* Host-side fault injection for tests: stall != 0 stops the server thread's heartbeat, so
   the device workers' idle waits run out (after heartbeat_timeout_s) and they stop with the
   error word set; 0 resumes it.  No device fault is involved. */
void pimqap_server_debug_stall_heartbeat(pimqap_server *s, int32_t stall);

/* ---------------------------------------------------------------- automatic beta */

/* The reference's automatic mode (autoSelectParameters, CPU_PIM.cpp:366-476): for beta0 =
   2^k, k = -30..1, five short trials (10 mega-iterations, every replica at beta0) average the
   final energies; the beta range is read off that curve with auto_lower / auto_higher.  All
   160 trials run as one batched launch.  Trial (k, t) is seeded from params.seed and 5k + t.
   Outputs: beta0 in internal units, deltaBeta, the 32 average energies (may be NULL) and the
   best energy / permutation any trial found (may be NULL; n entries). */
pimqap_status pimqap_auto_beta(const pimqap_instance *inst, const pimqap_params *params,
                               double *beta0_internal, double *delta_beta, double *avg_energy,
                               int64_t *best_energy, int32_t *best_perm);

/* Everything the reference's automatic mode prints and decides, for a drop-in of its log
   (CPU_PIM.cpp:373-476).  The trials run as in pimqap_auto_beta; in the reference they run one
   after another, so the first trial (in that order) whose tracked best reaches params.goal ends
   automatic mode: goal_trial is that trial and the later trials are ignored. */
#define PIMQAP_AUTO_STEPS 32
#define PIMQAP_AUTO_TRIALS 5
typedef struct pimqap_auto_report {
    double beta0_internal;      /* beta0 after automatic mode: maxBeta, or exp2(-30 + step) of
                                   the goal trial's step (:397, :420-422) */
    double delta_beta;          /* deltaBeta after automatic mode (1 when the goal ended it) */
    double min_beta, max_beta;  /* "Selecting minimum / maximum beta of" values (:449-461);
                                   0 when the goal ended automatic mode */
    int32_t min_beta_printed;   /* nonzero when the reference prints the minimum-beta line (it
                                   falls back to exp2(-30) silently otherwise, :454-456) */
    int32_t pad0;
    double avg_energy[PIMQAP_AUTO_STEPS];          /* "Average Energy" of each beta step */
    int64_t trial_best[PIMQAP_AUTO_STEPS * PIMQAP_AUTO_TRIALS];
                                /* best energy each trial's tracking saw (mega-iterations 0-9;
                                   the sweeps of the last one are not tracked, :293-362) */
    int32_t steps_printed;      /* beta steps whose "Beta:" line the reference prints */
    int32_t goal_trial;         /* -1, or the trial that reached the goal */
    int64_t best_energy;        /* best energy of any visited state over the trials used */
    int32_t *best_perm;         /* caller-provided, n entries (may be NULL) */
    pimqap_event *events;       /* caller-provided GROUP_BEST events of the trials used, in
                                   the reference's order (may be NULL) */
    int32_t event_capacity;     /* entries of events */
    int32_t event_count;        /* entries written */
    int64_t events_dropped;     /* events that did not fit */
    double device_ms;           /* device time of the trials */
} pimqap_auto_report;

pimqap_status pimqap_auto_beta_report(const pimqap_instance *inst, const pimqap_params *params,
                                      pimqap_auto_report *report);

/* ---------------------------------------------------------------- misc */

/* Diagnostic with no reference counterpart: measures the shared-memory read-modify-write
   bandwidth of the device (GB/s, reads + writes), the ceiling of the resident sweep. */
pimqap_status pimqap_probe_smem_bandwidth(int32_t device, double *gbs);

/* Diagnostic with no reference counterpart: evaluates the one-shot rule's binary32 weight
   function 2^x (x <= 0; exact bits of the solver's device code) on `count` inputs. */
pimqap_status pimqap_probe_weight_exp2(int32_t device, const float *x, float *y, int64_t count);

const char *pimqap_last_error(void);
const char *pimqap_version(void);

#ifdef __cplusplus
}
#endif
#endif
