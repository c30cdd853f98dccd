/*
 * ref_harness.cpp - appended after the reference's CPU-PIM/CPU_PIM.cpp (same translation
 * unit) by oracle/build_ref.sh.  It exports C entry points that drive the reference's own
 * readProblem() / setup() / doMegaItera() / threadToRun() over the reference's own globals.
 *
 * TEST INFRASTRUCTURE ONLY: tests use it to pin the oracle restatement to the reference,
 * and bench.py's reference arm uses it to time the reference's own sweep code.
 */
#include <chrono>
#include <cstring>
#include <streambuf>

namespace {
struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
};
NullBuf g_null;
std::streambuf *g_cout_buf = nullptr;
}  // namespace

#pragma GCC visibility push(default)
extern "C" {

int ref_maxn() { return MAXN; }
int ref_maxr() { return MAXNUMREPLICAS; }
int ref_maxt() { return MAXNUMTHREADS; }
int ref_has_shim() {
#ifdef PIMQAP_REF_NO_SHIM
    return 0;
#else
    return 1;
#endif
}

/* Silence the reference's progress lines on stdout (1) or restore them (0). */
void ref_quiet(int quiet) {
    if (!g_cout_buf) g_cout_buf = std::cout.rdbuf();
    std::cout.rdbuf(quiet ? static_cast<std::streambuf *>(&g_null) : g_cout_buf);
}

/* Instance from dense row-major arrays (F first, then D, as the file format orders them). */
int ref_load(int n, const int32_t *Fd, const int32_t *Dd) {
    if (n < 1 || n > MAXN) return 1;
    N = n;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            F[i * MAXN + j] = Fd[i * n + j];
            D[i * MAXN + j] = Dd[i * n + j];
        }
    return 0;
}

/* The reference's own file reader (CPU_PIM.cpp:79-107). */
int ref_read_file(const char *path) {
    inputFileName = path;
    return readProblem();
}

int ref_n() { return N; }

void ref_get_instance(int32_t *Fd, int32_t *Dd) {
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            Fd[i * N + j] = F[i * MAXN + j];
            Dd[i * N + j] = D[i * MAXN + j];
        }
}

/* setup() with fixed parameters (no automatic beta search).  beta0 is in the reference's
   internal units (the -b value times 1/ln 2, CPU_PIM.cpp:528). */
int ref_setup(int T, int R, int numitera, double beta0_internal, double delta_beta,
              uint64_t seed) {
    if (T < 1 || T > MAXNUMTHREADS || R < 1 || R > MAXNUMREPLICAS || numitera < 1) return 1;
    NUMTHREADS = T;
    NUMREPLICAS = R;
    NUMITERA = numitera;
    beta0 = beta0_internal;
    deltaBeta = delta_beta;
    automaticMode = false;
    goal = 0;
    goalPrint = 0;
    timeout = 0;
    singleBestE = 2147483647;
    pimqap_ref::g_seed = seed;
    pimqap_ref::g_shuffle_calls = 0;
    /* setup() initialises only the first R rank slots of each group; the slots past R keep
       their value, which is 0 in a fresh process.  Start every setup from that state. */
    std::memset(indexOfBetaOrder, 0, sizeof(indexOfBetaOrder));
    setup();
#ifndef PIMQAP_REF_NO_SHIM
    for (int t = 0; t < T; ++t) rng[t].bind_sweep((uint32_t)t, N, R, numitera);
#endif
    return 0;
}

/* For timing only: setup() of group 0 (the reference's own code), then groups 1..T-1 start
   as copies of group 0 with their own engines, seeded as setup() seeds them (CPU_PIM.cpp:130).
   The reference's setup() builds every group serially in O(T R n^3); copying keeps the bench's
   untimed set-up short while the timed threadToRun() path stays the reference's. */
int ref_setup_replicated(int T, int R, int numitera, double beta0_internal, double delta_beta,
                         uint64_t seed) {
    if (T < 1 || T > MAXNUMTHREADS) return 1;
    if (ref_setup(1, R, numitera, beta0_internal, delta_beta, seed)) return 1;
    std::random_device dev;
    for (int t = 1; t < T; ++t) {
        for (int l = 0; l < MAXNUMREPLICAS; ++l) {
            indexOfBetaOrder[t * MAXNUMREPLICAS + l] = indexOfBetaOrder[l];
            beta[t * MAXNUMREPLICAS + l] = beta[l];
        }
        for (int l = 0; l < R; ++l) {
            const size_t src = (size_t)l, dst = (size_t)t * MAXNUMREPLICAS + l;
            bestE[dst] = bestE[src];
            currentE[dst] = currentE[src];
            std::memcpy(&facilityOfLocation[dst * MAXN], &facilityOfLocation[src * MAXN], sizeof(int) * MAXN);
            std::memcpy(&locationOfFacility[dst * MAXN], &locationOfFacility[src * MAXN], sizeof(int) * MAXN);
            std::memcpy(&I[dst * MAXN * MAXN], &I[src * MAXN * MAXN], sizeof(int) * MAXN * MAXN);
        }
        timeSinceSwap[t] = timeSinceSwap[0];
        threadBestE[t] = threadBestE[0];
        rng[t] = std::mt19937(dev());
#ifndef PIMQAP_REF_NO_SHIM
        rng[t].bind_sweep((uint32_t)t, N, R, numitera);
#endif
    }
    NUMTHREADS = T;
    return 0;
}

void ref_set_goal(int g) { goal = g; }

/* megaiters iterations of threadToRun(t) for every group on one std::thread per group,
   exactly as main() launches them (CPU_PIM.cpp:666-674).  Returns wall seconds. */
double ref_run(int megaiters) {
    NUMMEGAITERA = megaiters;
    startTime = std::chrono::high_resolution_clock::now();
    auto t0 = std::chrono::steady_clock::now();
    for (int t = 0; t < NUMTHREADS; t++) threads[t] = std::thread([t]() { threadToRun(t); });
    for (int t = 0; t < NUMTHREADS; t++) threads[t].join();
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

void ref_domega(int t, int l) { doMegaItera(t, l); }

void ref_get_replica(int t, int l, int32_t *phi, int32_t *phiinv, int64_t *Iout, int64_t *E,
                     int64_t *bestEout, double *betaout) {
    const int rep = t * MAXNUMREPLICAS + l;
    for (int i = 0; i < N; ++i) {
        phi[i] = facilityOfLocation[rep * MAXN + i];
        phiinv[i] = locationOfFacility[rep * MAXN + i];
        for (int a = 0; a < N; ++a)
            Iout[i * N + a] = I[((size_t)rep * MAXN + i) * MAXN + a];
    }
    *E = currentE[rep];
    *bestEout = bestE[rep];
    *betaout = beta[rep];
}

/* order has MAXNUMREPLICAS entries (the whole slot range, junk slots included). */
void ref_get_group(int t, int32_t *order, int32_t *time_since_swap, int64_t *thread_best) {
    for (int l = 0; l < MAXNUMREPLICAS; ++l) order[l] = indexOfBetaOrder[t * MAXNUMREPLICAS + l];
    *time_since_swap = timeSinceSwap[t];
    *thread_best = threadBestE[t];
}

int64_t ref_single_best() { return singleBestE.load(); }

/* The reference CLI in process (argv[0] is the program name). */
int ref_main(int argc, char **argv) { return pimqap_ref_main(argc, argv); }

#ifndef PIMQAP_REF_NO_SHIM
/* The reference's own main() on the solver's Philox streams (see the CLI mode of
   ref_prelude.h): same flags, same files, same stdout, so its outputs can be compared line by
   line with the pimqap CLI run with --seed. */
int ref_cli(uint64_t seed, int argc, char **argv) {
    pimqap_ref::g_cli = true;
    pimqap_ref::g_cli_seed = seed;
    pimqap_ref::g_ctor_calls = 0;
    pimqap_ref::g_rng_base = reinterpret_cast<const char *>(&rng[0]);
    pimqap_ref::g_N = &N;
    pimqap_ref::g_R = &NUMREPLICAS;
    pimqap_ref::g_IT = &NUMITERA;
    pimqap_ref::g_T = &NUMTHREADS;
    pimqap_ref::g_main = std::this_thread::get_id();
    return pimqap_ref_main(argc, argv);
}
#endif

}  // extern "C"
#pragma GCC visibility pop
