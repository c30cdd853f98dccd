// pimqap_host.cpp - host runtime behind the C ABI (include/pimqap.h).
//
// Reference mapping (CPU-PIM/CPU_PIM.cpp):
//   pimqap_read_problem      readProblem()                      :79-107
//   pimqap_solver_create     setup()                            :109-193
//   pimqap_solver_run        threadToRun() mega-iteration loop  :292-364
//   pimqap_solve             main() after flag parsing          :612-684
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "pimqap.h"
#include "pimqap_internal.h"
#include "pimqap_plan.h"
#include "pimqap_events.h"

using pimqap::SolveDev;

namespace {
thread_local std::string g_error;
}  // namespace

void pimqap::set_last_error(const char *msg) { g_error = msg; }

namespace pimqap {
namespace detail {

pimqap_status fail(pimqap_status st, const std::string &msg) {
    g_error = msg;
    return st;
}

void trace(const char *phase) {
    static const bool on = std::getenv("PIMQAP_TRACE") != nullptr;
    if (!on) return;
    static thread_local auto last = std::chrono::steady_clock::now();
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "[pimqap] %-32s %9.3f ms\n", phase,
                 std::chrono::duration<double, std::milli>(now - last).count());
    last = now;
}



// ------------------------------------------------------------------ initial permutations

void shuffle_group(ShuffleEngine &eng, int n, int32_t *perm) {
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int i = 0; i < n; ++i) {
        std::uniform_int_distribution<ShuffleEngine::result_type> distN(0, n - 1);
        const int j = (int)distN(eng);
        if (i != j) std::swap(perm[i], perm[j]);
    }
}

// Initial permutations of all groups (CPU_PIM.cpp:134-162); all replicas of a group share
// their group's permutation.
std::vector<int32_t> initial_perms(int n, int T, uint64_t seed) {
    std::vector<int32_t> perms((size_t)T * n);
    ShuffleEngine eng;
    eng.seed = seed;
    for (int t = 0; t < T; ++t) shuffle_group(eng, n, perms.data() + (size_t)t * n);
    return perms;
}

// ------------------------------------------------------------------ instance analysis


// Force-matrix width: |I[i][a]| <= sum_j |D_ij||F_a,phi(j)| + |D_ji||F_phi(j),a| is bounded by
// the rearrangement inequality (both rows sorted descending); a delta adds at most
// 4 max|I| + 16 max|D| max|F|.  int32 is used when that bound is below 2^31.
InstanceInfo analyse(int n, const int32_t *F, const int32_t *D) {
    InstanceInfo info;
    bool sym = true;
    long double A = 0, B = 0;
    for (int i = 0; i < n && sym; ++i)
        for (int j = 0; j < n; ++j)
            if (D[i * n + j] != D[j * n + i] || F[i * n + j] != F[j * n + i]) {
                sym = false;
                break;
            }
    info.symmetric = sym;
    info.binary_flow = true;
    info.dist16 = true;
    info.dmin = info.dmax = D[0];
    info.fmin = info.fmax = F[0];
    for (int k = 0; k < n * n; ++k) {
        if (F[k] != 0 && F[k] != 1) info.binary_flow = false;
        if (D[k] < -32768 || D[k] > 32767) info.dist16 = false;
        info.dmin = std::min<int64_t>(info.dmin, D[k]);
        info.dmax = std::max<int64_t>(info.dmax, D[k]);
        info.fmin = std::min<int64_t>(info.fmin, F[k]);
        info.fmax = std::max<int64_t>(info.fmax, F[k]);
    }
    if (info.binary_flow) {   // clique of unit flows on a prefix of the facilities?
        int A = 0;
        while (A < n && [&] { for (int b = 0; b < n; ++b) if (F[A * n + b]) return true; return false; }()) ++A;
        bool ok = A >= 2 && A < n;
        for (int a = 0; a < n && ok; ++a) {
            ok = D[a * n + a] == 0;
            for (int b = 0; b < n && ok; ++b) ok = F[a * n + b] == ((a != b && a < A && b < A) ? 1 : 0);
        }
        info.clique = ok ? A : 0;
    }
    std::vector<long double> rD(n, 0), cD(n, 0);
    long double rFmax = 0, cFmax = 0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const long double d = std::fabs((long double)D[i * n + j]);
            const long double f = std::fabs((long double)F[i * n + j]);
            A = std::max(A, d);
            B = std::max(B, f);
            rD[i] += d;
            cD[j] += d;
        }
    for (int a = 0; a < n; ++a) {
        long double r = 0, c = 0;
        for (int b = 0; b < n; ++b) {
            r = std::max(r, std::fabs((long double)F[a * n + b]));
            c = std::max(c, std::fabs((long double)F[b * n + a]));
        }
        rFmax = std::max(rFmax, r);
        cFmax = std::max(cFmax, c);
    }
    long double imax = 0;
    for (int i = 0; i < n; ++i) imax = std::max(imax, rD[i] * rFmax + cD[i] * cFmax);
    auto delta_bound = [&](long double im) { return 4 * im + 16 * A * B; };
    const long double lim32 = 2147483647.0L, lim64 = 4.6e18L;
    if (delta_bound(imax) >= lim32) {
        // tighter: sorted rows (rearrangement inequality)
        std::vector<std::vector<long double>> Dr(n), Dc(n), Fr(n), Fc(n);
        for (int i = 0; i < n; ++i) {
            Dr[i].resize(n); Dc[i].resize(n); Fr[i].resize(n); Fc[i].resize(n);
            for (int j = 0; j < n; ++j) {
                Dr[i][j] = std::fabs((long double)D[i * n + j]);
                Dc[i][j] = std::fabs((long double)D[j * n + i]);
                Fr[i][j] = std::fabs((long double)F[i * n + j]);
                Fc[i][j] = std::fabs((long double)F[j * n + i]);
            }
            std::sort(Dr[i].rbegin(), Dr[i].rend());
            std::sort(Dc[i].rbegin(), Dc[i].rend());
            std::sort(Fr[i].rbegin(), Fr[i].rend());
            std::sort(Fc[i].rbegin(), Fc[i].rend());
        }
        long double tight = 0;
        for (int i = 0; i < n; ++i)
            for (int a = 0; a < n; ++a) {
                long double s = 0;
                for (int k = 0; k < n; ++k) s += Dr[i][k] * Fr[a][k] + Dc[i][k] * Fc[a][k];
                tight = std::max(tight, s);
            }
        imax = std::min(imax, tight);
    }
    long double ebound = 0;
    for (int i = 0; i < n; ++i) ebound += rD[i] * rFmax;
    if (delta_bound(imax) < lim32) info.bits_needed = 32;
    else if (delta_bound(imax) < lim64 && ebound < lim64) info.bits_needed = 64;
    else info.bits_needed = 0;
    return info;
}

int round_up(int x, int m) { return (x + m - 1) / m * m; }

}  // namespace detail
}  // namespace pimqap

using namespace pimqap::detail;

// ------------------------------------------------------------------ device block reuse

namespace {

// A finished handle's device block (up to kKeepBytes) is kept for the next handle on the same
// device, so back-to-back solves make no cudaMalloc / cudaFree: both take the driver's
// allocation locks and cudaFree waits for the whole device, which on a busy host has cost up
// to 0.6 s in a solve of 0.36 s.  One block per device; larger blocks are freed as before.
// Every byte of a block is rewritten by the next solve's set-up (head uploaded, tail cleared).
constexpr size_t kKeepBytes = 256ull << 20;
constexpr int kKeepDevices = 64;
struct KeptBlock {
    void *p = nullptr;
    size_t bytes = 0;
};
std::mutex g_keep_mu;
KeptBlock g_keep[kKeepDevices];

// A block of at least `bytes` on the current device (`device`): the kept one when it is big
// enough, else a new allocation.  *got is the block's real size.
cudaError_t block_acquire(int device, size_t bytes, void **p, size_t *got) {
    if (device >= 0 && device < kKeepDevices) {
        std::lock_guard<std::mutex> lk(g_keep_mu);
        KeptBlock &k = g_keep[device];
        if (k.p && k.bytes >= bytes) {
            *p = k.p;
            *got = k.bytes;
            k = KeptBlock{};
            return cudaSuccess;
        }
    }
    *got = bytes;
    return cudaMalloc(p, bytes);
}

// Returns a block no work is pending on: kept when it is small enough and larger than the
// block kept now (which is freed instead), else freed.
void block_release(int device, void *p, size_t bytes) {
    if (!p) return;
    if (bytes <= kKeepBytes && device >= 0 && device < kKeepDevices) {
        void *drop = p;
        {
            std::lock_guard<std::mutex> lk(g_keep_mu);
            KeptBlock &k = g_keep[device];
            if (!k.p || k.bytes < bytes) {
                drop = k.p;
                k = KeptBlock{p, bytes};
            }
        }
        if (drop) cudaFree(drop);
        return;
    }
    cudaFree(p);
}

}  // namespace

// ------------------------------------------------------------------ solver object

struct pimqap_solver {
    pimqap_params p{};
    int n = 0, T = 0, R = 0, cap = 0, spe = 0;
    int bits = 32, cl = 1, threads = 256;
    bool sym = false, bin = false, pair = false, pipe = false;
    bool persistent = false;   // one persistent launch per run call (solve_kernel)
    size_t smem = 0;
    int device = 0;
    volatile int32_t *kill = nullptr;   // mapped host word of the persistent launch (timeout)
    int64_t launches = 0;               // sweep-kernel launches so far
    cudaGraphExec_t solve_graph = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    void *dmem = nullptr;
    size_t dbytes = 0;
    SolveDev dev{};
    cudaGraphExec_t graph = nullptr;
    int graph_epochs = 0;
    int64_t megaiters_done = 0;
    double device_ms = 0;
    bool stopped_goal = false;
    int64_t h2d = 0, d2h = 0;   // bytes copied over PCIe by this solver
    double beta0_used = 0, ratio_used = 0;
    std::unique_ptr<pimqap::detail::EventBuffer> events;   // params.event_capacity > 0
    unsigned long long start_ns = 0;                        // %globaltimer at setup

    ~pimqap_solver() {
        events.reset();
        if (graph) cudaGraphExecDestroy(graph);
        if (solve_graph) cudaGraphExecDestroy(solve_graph);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) {
            cudaStreamSynchronize(stream);   // nothing in flight on the block it gives back
            cudaStreamDestroy(stream);
        }
        block_release(device, dmem, dbytes);
        if (kill) cudaFreeHost(const_cast<int32_t *>(kill));
    }
};

namespace pimqap {
namespace detail {

pimqap_status check_params(const pimqap_instance *inst, const pimqap_params *p) {
    if (!inst || !p) return fail(PIMQAP_ERR_ARG, "null instance or params");
    if (inst->n < 1 || inst->n > PIMQAP_MAX_N)
        return fail(PIMQAP_ERR_ARG, "n must be in [1, " + std::to_string(PIMQAP_MAX_N) + "]");
    if (!inst->flow || !inst->dist) return fail(PIMQAP_ERR_ARG, "null flow or dist");
    if (p->replicas < 1 || p->replicas > PIMQAP_MAX_REPLICAS)
        return fail(PIMQAP_ERR_ARG, "replicas must be in [1, " + std::to_string(PIMQAP_MAX_REPLICAS) + "]");
    if (p->groups < 1 || p->groups > PIMQAP_MAX_GROUPS)
        return fail(PIMQAP_ERR_ARG, "groups must be in [1, " + std::to_string(PIMQAP_MAX_GROUPS) + "]");
    if (p->sweeps_per_exchange < 1) return fail(PIMQAP_ERR_ARG, "sweeps_per_exchange must be >= 1");
    if (p->rank_slots != 0 && (p->rank_slots < p->replicas || p->rank_slots > 4096))
        return fail(PIMQAP_ERR_ARG, "rank_slots must be 0 or in [replicas, 4096]");
    if (!(p->beta_max > 0) || !std::isfinite(p->beta_max))
        return fail(PIMQAP_ERR_ARG, "beta_max must be a positive finite number");
    if (!(p->beta_ratio > 0) || !std::isfinite(p->beta_ratio))
        return fail(PIMQAP_ERR_ARG, "beta_ratio must be a positive finite number");
    if (p->max_megaiters < 0) return fail(PIMQAP_ERR_ARG, "max_megaiters must be >= 0");
    if (!(p->timeout_s >= 0) || !std::isfinite(p->timeout_s))   // -s (CPU_PIM.cpp:350-357)
        return fail(PIMQAP_ERR_ARG, "timeout_s must be a finite number >= 0 (0 = no timeout)");
    if (p->event_capacity < 0 || p->event_perm_capacity < 0)
        return fail(PIMQAP_ERR_ARG, "event capacities must be >= 0");
    if (p->compact_instance != 0 && p->compact_instance != 1)
        return fail(PIMQAP_ERR_ARG, "compact_instance must be 0 or 1");
    if (p->active_facilities != 0 && (p->active_facilities < 2 || p->active_facilities >= inst->n))
        return fail(PIMQAP_ERR_ARG, "active_facilities must be 0 or in [2, n)");
    if (p->update_rule != PIMQAP_RULE_SEQUENTIAL && p->update_rule != PIMQAP_RULE_ONE_SHOT)
        return fail(PIMQAP_ERR_ARG, "update_rule must be 0 (sequential) or 1 (one-shot)");
    if (p->update_rule == PIMQAP_RULE_ONE_SHOT && p->active_facilities != 0)
        return fail(PIMQAP_ERR_ARG, "active_facilities applies to the sequential rule only");
    if (p->force_bits != 0 && p->force_bits != 32 && p->force_bits != 64)
        return fail(PIMQAP_ERR_ARG, "force_bits must be 0, 32 or 64");
    if (p->threads_per_block != 0 && p->threads_per_block != 64 && p->threads_per_block != 128 &&
        p->threads_per_block != 256 && !(p->threads_per_block == 512 && p->update_rule == PIMQAP_RULE_ONE_SHOT) &&
        !(p->threads_per_block == 32 && inst->n <= 128 && p->update_rule == PIMQAP_RULE_SEQUENTIAL))
        return fail(PIMQAP_ERR_ARG, "threads_per_block must be 0, 64, 128 or 256 (512 with the one-shot rule, "
                                    "32 with the sequential rule for n <= 128)");
    if (p->cluster_size != 0 && p->cluster_size != 1 && p->cluster_size != 2 && p->cluster_size != 4)
        return fail(PIMQAP_ERR_ARG, "cluster_size must be 0, 1, 2 or 4");
    if (p->replica_pairing < 0 || p->replica_pairing > 2)
        return fail(PIMQAP_ERR_ARG, "replica_pairing must be 0 (automatic), 1 (off) or 2 (on)");
    if (p->sweep_pipeline < 0 || p->sweep_pipeline > 2)
        return fail(PIMQAP_ERR_ARG, "sweep_pipeline must be 0 (automatic), 1 (off) or 2 (on)");
    if (p->launch_mode < 0 || p->launch_mode > 2)
        return fail(PIMQAP_ERR_ARG, "launch_mode must be 0 (automatic), 1 (a launch per mega-iteration) or "
                                    "2 (one persistent launch)");
    if (p->tensor_update < 0 || p->tensor_update > 3)
        return fail(PIMQAP_ERR_ARG, "tensor_update must be 0 (automatic), 1 (integer CUDA cores), 2 (mma.sync) "
                                    "or 3 (tcgen05)");
    if (p->tensor_update == 2 && p->update_rule != PIMQAP_RULE_ONE_SHOT)
        return fail(PIMQAP_ERR_ARG, "tensor_update 2 (mma.sync) applies to the one-shot rule only");
    if (p->oneshot_weights < 0 || p->oneshot_weights > 1)
        return fail(PIMQAP_ERR_ARG, "oneshot_weights must be 0 (CUDA's exp2f, as the reference) or 1 (this "
                                    "library's own 2^x)");
    return PIMQAP_OK;
}


// ------------------------------------------------------------------ per-instance plan + staging

pimqap_status open_device(int device, int *maxsm) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(PIMQAP_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(PIMQAP_ERR_ARG, "bad device ordinal");
    PQ_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    PQ_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return fail(PIMQAP_ERR_NO_DEVICE, "the kernels are built for sm_100a only");
    PQ_CUDA(pimqap::prepare_kernels());
    *maxsm = (int)prop.sharedMemPerBlockOptin;
    return PIMQAP_OK;
}

pimqap_status plan_instance(const pimqap_instance *inst, const pimqap_params *params, size_t maxsm,
                            int want_cluster, Plan *out, const InstanceInfo *known) {
    const int n = inst->n;
    const InstanceInfo info = known ? *known : analyse(n, inst->flow, inst->dist);
    if (info.bits_needed == 0 && params->force_bits == 0)
        return fail(PIMQAP_ERR_RANGE, "instance values can overflow int64 force matrices");
    Plan P;
    P.n = n;
    P.T = params->groups;
    P.R = params->replicas;
    P.cap = params->rank_slots ? params->rank_slots : std::max(params->replicas, 10);
    P.spe = params->sweeps_per_exchange;
    P.sym = info.symmetric;
    P.bits = params->force_bits ? params->force_bits : info.bits_needed;
    const int isz = P.bits / 8, vec = 16 / isz;
    P.npad = round_up(n, 4);
    P.lds = P.npad;
    if ((P.lds / vec) % 2 == 0) P.lds += vec;
    P.threads = params->threads_per_block ? params->threads_per_block
                                          : (n <= 64 ? 64 : (n <= 128 ? 128 : 256));
    auto rows_per_cta = [&](int cl) { return round_up((n + cl - 1) / cl, 4); };
    if (params->update_rule == PIMQAP_RULE_ONE_SHOT) {
        P.os_own_exp2 = params->oneshot_weights == 1;
        // the one-shot epoch: odd row stride (column reads by 32 lanes hit 32 banks), the
        // smallest cluster that holds its rows with a force-update chunk of 32, 16, 8 or 4 swaps,
        // preferring the layout whose peers push the columns the proposals need
        P.lds = P.npad + 1;
        P.cl = 0;
        // the force update on the tensor cores when fp16 holds every factor exactly (at most 2048
        // in magnitude: 2 dD for symmetric instances, dD otherwise, and dF) and no fp32 sum can
        // reach 2^24 (n / 2 swaps x 2 terms x |dD| |dF|)
        const int64_t dr = info.dmax - info.dmin, fr = info.fmax - info.fmin;
        const bool exact = (info.symmetric ? 2 * dr : dr) <= 2048 && fr <= 2048 &&
                           (int64_t)n * dr * fr < (int64_t)1 << 24 && params->compact_instance == 0;
        const int want = params->tensor_update;              // 0 auto, 1 CUDA cores, 2 mma.sync, 3 tcgen05
        if (want >= 2 && !exact)
            return fail(PIMQAP_ERR_ARG, "tensor_update 2 / 3 needs an instance whose force-update factors fp16 "
                                        "holds exactly (2 dD or dD, and dF, at most 2048 in magnitude) with "
                                        "n |dD| |dF| below 2^24");
        // tcgen05 (M = 128 rows per CTA, N <= 256 columns, four TMEM lane quarters read by
        // warps 0-3 mod 4): at most 128 rows per CTA, n <= 256, a multiple of 128 threads
        const int thr = params->threads_per_block;
        auto os_mode = [&](int cl) {
            if (!exact || want == 1) return 0;
            const bool tc_ok = rows_per_cta(cl) <= 128 && n <= 256 && (thr == 0 || thr % 128 == 0);
            if (want == 3) return tc_ok ? 2 : -1;
            if (want == 2) return 1;
            return tc_ok ? 2 : 1;
        };
        for (int cl : {1, 2, 4}) {
            if (want_cluster && cl != want_cluster) continue;
            const int mode = os_mode(cl);
            if (mode < 0) continue;
            for (int xcol = (cl > 1 ? 1 : 0); xcol >= 0 && !P.cl; --xcol)
                for (int pc : {32, 16, 8, 4}) {
                    const size_t sm = pimqap::epoch_smem_bytes_os(n, rows_per_cta(cl), P.lds, cl, P.bits, pc,
                                                                  P.sym, xcol != 0, mode);
                    if (sm <= maxsm) {
                        P.cl = cl;
                        P.os_chunk = pc;
                        P.os_xcol = xcol;
                        P.os_mma = mode;
                        P.smem = sm;
                        break;
                    }
                }
            if (P.cl) break;
        }
        if (!P.cl && want == 3)
            return fail(PIMQAP_ERR_ARG, "tensor_update 3 (tcgen05) needs at most 128 rows per CTA, n <= 256 and a "
                                        "multiple of 128 threads per block");
        if (!P.cl) return fail(PIMQAP_ERR_ARG, "force matrix does not fit the requested cluster size");
        P.rpc = rows_per_cta(P.cl);
        P.ldm = std::max(P.npad, P.cl * P.rpc);
        if (!params->threads_per_block) P.threads = P.rpc > 64 ? 512 : (P.rpc > 32 ? 256 : 128);
        if (P.os_mma == 2) {
            // Each CTA of the tcgen05 form holds `tcols` of its SM's 512 tensor-memory columns
            // from start to end, and its allocation waits while they are taken; a CTA of a
            // cluster waiting there for a CTA whose peer waits the same way elsewhere would wait
            // for good.  So the shared-memory request is raised until at most 512 / tcols CTAs
            // fit on one SM, and no allocation ever waits.
            int dev = 0, smpm = 0, resv = 0;
            PQ_CUDA(cudaGetDevice(&dev));
            PQ_CUDA(cudaDeviceGetAttribute(&smpm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
            PQ_CUDA(cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, dev));
            const int allowed = 512 / pimqap::os_tmem_columns(n);
            if (smpm / ((int)P.smem + resv) > allowed)
                P.smem = (size_t)round_up(smpm / (allowed + 1) - resv + 16, 16);   // allowed + 1 do not fit
        }
    }
    if (!P.os_chunk) {
    P.cl = 0;
    for (int cl : {1, 2, 4}) {
        if (want_cluster && cl != want_cluster) continue;
        if (pimqap::epoch_smem_bytes(n, rows_per_cta(cl), P.lds, cl, P.bits) <= maxsm) {
            P.cl = cl;
            break;
        }
    }
    if (!P.cl) return fail(PIMQAP_ERR_ARG, "force matrix does not fit the requested cluster size");
    P.rpc = rows_per_cta(P.cl);
    // D / F rows are read in 16-byte chunks up to column cl * rpc
    P.ldm = std::max(P.npad, P.cl * P.rpc);
    P.smem = pimqap::epoch_smem_bytes(n, P.rpc, P.lds, P.cl, P.bits);
    }
    // binary flows and int16 distances: the instance itself fits next to the force rows
    if (info.symmetric && info.binary_flow && info.dist16 && P.bits == 32 && !P.os_chunk &&
        (params->compact_instance == 0 || params->active_facilities > 0)) {
        const size_t sb = pimqap::epoch_smem_bytes_bin(n, P.rpc, P.lds, P.cl, false);
        if (sb <= maxsm) {
            P.bin = true;
            P.smem_bin = sb;
        }
        // its 16-swap rewrite of the rows on the tcgen05 tensor cores where fp16 holds every
        // factor exactly (2 (D[k][j] - D[k][i]) at most 2048 in magnitude: a distance range of at
        // most 1024; flow differences are -1, 0 or 1; 16 terms stay below 2^24), an M = 128 MMA
        // covers a CTA's rows (n <= 256) and whole warp quarters read them back (a multiple of
        // 128 threads); not with clique moves (no swap log)
        const int want = params->tensor_update;
        const bool tc_ok = P.bin && params->active_facilities == 0 && info.dmax - info.dmin <= 1024 &&
                           P.rpc <= 128 && n <= 256 && P.threads % 128 == 0;
        if (tc_ok && want != 1) {
            size_t st = pimqap::epoch_smem_bytes_bin(n, P.rpc, P.lds, P.cl, true);
            // each CTA holds `tcols` of its SM's 512 tensor-memory columns for its whole epoch and
            // its allocation waits while they are taken; a CTA of a cluster waiting there for a
            // CTA whose peer waits the same way elsewhere would wait for good.  So the shared-memory
            // request is raised until at most 512 / tcols CTAs fit on an SM.
            const int tcn = round_up(n, 16);
            const int tcols = tcn <= 32 ? 32 : (tcn <= 64 ? 64 : (tcn <= 128 ? 128 : 256));
            const int allowed = 512 / tcols;
            int dev = 0, smpm = 0, resv = 0;
            PQ_CUDA(cudaGetDevice(&dev));
            PQ_CUDA(cudaDeviceGetAttribute(&smpm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
            PQ_CUDA(cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, dev));
            if (smpm / ((int)st + resv) > allowed) st = (size_t)round_up(smpm / (allowed + 1) - resv + 16, 16);
            if (st <= maxsm) {
                P.bin_tc = true;
                P.smem_bin = st;
            }
        }
    }
    if (params->tensor_update == 3 && params->update_rule != PIMQAP_RULE_ONE_SHOT && !P.bin_tc)
        return fail(PIMQAP_ERR_ARG, "tensor_update 3 (tcgen05) with the sequential rule needs the binary-flow "
                                    "kernel (symmetric 0/1 flows, int16 distances, int32 forces), a distance "
                                    "range of at most 1024, no clique moves, n <= 256, a multiple of 128 "
                                    "threads per block and a layout that fits");
    if (params->active_facilities > 0) {   // the tai256c program's moves (CPU_PIM_tai256c.cpp)
        if (!P.bin || !info.symmetric || info.clique != params->active_facilities)
            return fail(PIMQAP_ERR_ARG, "active_facilities needs a symmetric instance whose flows are a clique of "
                                        "unit flows on facilities 0..active_facilities-1 (zero diagonals, "
                                        "distances within int16, int32 forces)");
        P.act = params->active_facilities;
    }
    const size_t reps = (size_t)P.T * P.R, nn = (size_t)n * P.ldm;
    // head: everything uploaded from the host; tail: state that starts at zero
    P.head = 4 * carve_size(nn * 4) + 2 * carve_size((size_t)n * 4) + carve_size(reps * n * 4) +
             carve_size(reps * 8) + carve_size((size_t)P.T * P.cap * 4) + carve_size((size_t)P.T * 8) +
             4 * carve_size(8);
    P.tail = carve_size(reps * (size_t)n * P.npad * isz) + carve_size(reps * n * 4) + 3 * carve_size(reps * 8) +
             3 * carve_size((size_t)P.T * 8) + 5 * carve_size(8);
    P.total = P.head + P.tail;
    P.h2d_bytes = (int64_t)P.head;
    *out = P;
    return PIMQAP_OK;
}

pimqap_status plan_pairing(const pimqap_instance *inst, const pimqap_params *params, size_t maxsm,
                           Plan *P) {
    // Automatic mode does not pair: with one replica per update chain the throughput is set by
    // the chain's latency, and on the n = 256 workload two chains per 4-CTA cluster measured
    // 2.64e9 proposals/s against 2.95e9 for one chain per 2-CTA cluster.
    if (params->replica_pairing != 2) return PIMQAP_OK;
    // the unpaired plan may use the generic kernel where the binary-flow layout needs a larger
    // cluster than the generic one: every cluster size is tried for the pair
    if (!P->os_chunk && (int64_t)P->T * P->R >= 2) {
        for (int cl : {1, 2, 4}) {
            if (cl < P->cl || (params->cluster_size && cl != params->cluster_size)) continue;
            Plan Q;
            if (plan_instance(inst, params, maxsm, cl, &Q) != PIMQAP_OK || !Q.bin) continue;
            const size_t sp = pimqap::epoch_smem_bytes_bin_pair(Q.n, Q.rpc, Q.lds, cl);
            if (sp > maxsm) continue;
            Q.pair = true;
            Q.smem_bin = sp;
            *P = Q;
            return PIMQAP_OK;
        }
    }
    return fail(PIMQAP_ERR_ARG, "replica_pairing = 2 needs the binary-flow kernel (symmetric 0/1 flows, "
                                "int16 distances, int32 forces, sequential rule, at least two replicas) "
                                "and a paired layout that fits the cluster size");
}

void carve_instance(const Plan &P, char *head, char *tail, SolveDev *out) {
    const int n = P.n, T = P.T, R = P.R, cap = P.cap;
    const size_t reps = (size_t)T * R, nn = (size_t)n * P.ldm;
    SolveDev d{};
    d.n = n; d.R = R; d.T = T; d.cap = cap; d.spe = P.spe;
    d.act = P.act;
    d.os_chunk = P.os_chunk;
    d.os_xcol = P.os_xcol;
    d.os_mma = P.os_mma;
    d.os_own_exp2 = P.os_own_exp2;
    d.bin_tc = (P.bin_tc && !P.pair && !P.pipe) ? 1 : 0;
    d.ldg = P.npad; d.lds = P.lds; d.ldm = P.ldm; d.rpc = P.rpc;
    char *cur = head;
    d.D = carve<int32_t>(cur, nn);
    d.DT = carve<int32_t>(cur, nn);
    d.F = carve<int32_t>(cur, nn);
    d.FT = carve<int32_t>(cur, nn);
    d.Ddiag = carve<int32_t>(cur, n);
    d.Fdiag = carve<int32_t>(cur, n);
    d.phi = carve<int32_t>(cur, reps * n);
    d.beta = carve<double>(cur, reps);
    d.order = carve<int32_t>(cur, (size_t)T * cap);
    d.group_best = carve<int64_t>(cur, T);
    d.single_best = carve<int64_t>(cur, 1);
    d.stop_epoch = carve<int32_t>(cur, 1);
    d.target_epoch = carve<int64_t>(cur, 1);
    d.target_ns = carve<unsigned long long>(cur, 1);
    cur = tail;
    d.I = carve<char>(cur, reps * (size_t)n * P.npad * (P.bits / 8));
    d.best_phi = carve<int32_t>(cur, reps * n);
    d.E = carve<int64_t>(cur, reps);
    d.bestE = carve<int64_t>(cur, reps);
    d.accepts = carve<unsigned long long>(cur, reps);
    d.tss = carve<int32_t>(cur, T);
    d.finish = carve<unsigned int>(cur, T);
    d.epoch = carve<int32_t>(cur, T);
    d.start_ns = carve<unsigned long long>(cur, 1);
    d.error = carve<int32_t>(cur, 1);
    d.epoch_all = carve<int32_t>(cur, 1);
    d.finish_all = carve<unsigned int>(cur, 1);
    d.run_end = carve<int32_t>(cur, 1);
    d.kill = nullptr;
    *out = d;
}

// setup() for one instance on the host side (CPU_PIM.cpp:109-162): writes the padded
// matrices, transposes, diagonals, initial permutations, beta ladder, rank slots and the
// sentinels into `mirror`, a host image of the instance's head region (P.head bytes) laid out
// as carve_instance lays out the device head.
void fill_head(const pimqap_instance *inst, const pimqap_params *params, const Plan &P,
               char *mirror) {
    SolveDev h;
    carve_instance(P, mirror, mirror, &h);   // head pointers into the mirror
    const int n = P.n, T = P.T, R = P.R, cap = P.cap, ldm = P.ldm;
    const size_t reps = (size_t)T * R;
    std::memset(mirror, 0, P.head);
    int32_t *Dp = const_cast<int32_t *>(h.D), *DT = const_cast<int32_t *>(h.DT);
    int32_t *Fp = const_cast<int32_t *>(h.F), *FT = const_cast<int32_t *>(h.FT);
    int32_t *Dd = const_cast<int32_t *>(h.Ddiag), *Fd = const_cast<int32_t *>(h.Fdiag);
    for (int i = 0; i < n; ++i) {
        Dd[i] = inst->dist[i * n + i];
        Fd[i] = inst->flow[i * n + i];
        for (int j = 0; j < n; ++j) {
            Dp[(size_t)i * ldm + j] = inst->dist[i * n + j];
            Fp[(size_t)i * ldm + j] = inst->flow[i * n + j];
            DT[(size_t)i * ldm + j] = inst->dist[j * n + i];
            FT[(size_t)i * ldm + j] = inst->flow[j * n + i];
        }
    }
    const std::vector<int32_t> perms = initial_perms(n, T, params->seed);
    for (int t = 0; t < T; ++t)
        for (int l = 0; l < R; ++l)
            std::memcpy(&h.phi[((size_t)t * R + l) * n], &perms[(size_t)t * n], sizeof(int32_t) * n);
    // beta ladder (CPU_PIM.cpp:111-119); -b is given in natural units and stored x 1/ln 2 (:528)
    const double beta0 = params->beta_internal ? params->beta_max : params->beta_max * 1.44269504089;
    for (int t = 0; t < T; ++t) {
        double running = beta0;
        for (int l = R - 1; l >= 0; --l) {
            h.beta[(size_t)t * R + l] = running;
            running /= params->beta_ratio;
        }
    }
    for (int t = 0; t < T; ++t)
        for (int l = 0; l < R; ++l) h.order[(size_t)t * cap + l] = l;
    for (int t = 0; t < T; ++t) h.group_best[t] = pimqap::kNoBest;
    *h.single_best = pimqap::kNoBest;
    *h.stop_epoch = pimqap::kNoStop;
    *h.target_epoch = std::numeric_limits<int64_t>::max();
    *h.target_ns = ~0ull;
    (void)reps;
}

pimqap_status stage_instance(const pimqap_instance *inst, const pimqap_params *params,
                             const Plan &P, char *base, SolveDev *out, cudaStream_t q,
                             std::vector<std::vector<char>> &keep, const EventLink *ev) {
    keep.emplace_back(P.head, 0);
    char *mirror = keep.back().data();
    fill_head(inst, params, P, mirror);
    carve_instance(P, base, base + P.head, out);
    out->goal = params->goal;
    out->seed = params->seed;
    if (ev) out->ev = *ev;
    PQ_CUDA(cudaMemcpyAsync(base, mirror, P.head, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemsetAsync(base + P.head, 0, P.tail, q));
    PQ_CUDA(pimqap::launch_setup(*out, P.bits, q));
    return PIMQAP_OK;
}

}  // namespace detail
}  // namespace pimqap

extern "C" {

void pimqap_default_params(pimqap_params *p) {
    std::memset(p, 0, sizeof(*p));
    p->replicas = 10;               // MAXNUMREPLICAS (CPU_PIM.cpp:23-24)
    p->groups = 20;                 // MAXNUMTHREADS (:26-27)
    p->sweeps_per_exchange = 4;     // NUMITERA (:19)
    p->rank_slots = 0;
    p->max_megaiters = 2147483647;  // NUMMEGAITERA (:21)
    p->beta_max = std::exp2(-12.0) * 0.69314718055994530942;  // beta0 = 2^-12 internal (:29)
    p->beta_ratio = 1.2;            // deltaBeta (:31)
    p->goal = 0;                    // goal (:48)
    p->timeout_s = 0;
    p->seed = 1;
    p->device = 0;
    p->auto_lower = 0.1;            // lowerBetaProportion (:33)
    p->auto_higher = 0.9;           // higherBetaProportion (:34)
}

const char *pimqap_last_error(void) { return g_error.c_str(); }
const char *pimqap_version(void) { return "pimqap 0.1 (sm_100a)"; }

pimqap_status pimqap_read_problem(const char *path, int32_t max_n, int32_t *n_out,
                                  int32_t *flow, int32_t *dist) {
    if (!path || !n_out) return fail(PIMQAP_ERR_ARG, "null path or n");
    std::ifstream in(path);
    if (!in.is_open()) return fail(PIMQAP_ERR_IO, std::string("could not open the file (") + path + ")");
    long long n = 0;
    if (!(in >> n) || n < 1) return fail(PIMQAP_ERR_IO, "could not read n");
    if (n > max_n || n > PIMQAP_MAX_N)
        return fail(PIMQAP_ERR_ARG, "N exceeded MAXN (" + std::to_string(std::min<long long>(max_n, PIMQAP_MAX_N)) + ")");
    *n_out = (int32_t)n;
    if (!flow && !dist) return PIMQAP_OK;
    if (!flow || !dist) return fail(PIMQAP_ERR_ARG, "flow and dist must both be given");
    for (long long k = 0; k < n * n; ++k) {
        long long v;
        if (!(in >> v)) return fail(PIMQAP_ERR_IO, "flow matrix truncated");
        flow[k] = (int32_t)v;
    }
    for (long long k = 0; k < n * n; ++k) {
        long long v;
        if (!(in >> v)) return fail(PIMQAP_ERR_IO, "distance matrix truncated");
        dist[k] = (int32_t)v;
    }
    return PIMQAP_OK;
}

pimqap_status pimqap_load_file(const char *path, pimqap_instance *inst) {
    if (!inst) return fail(PIMQAP_ERR_ARG, "null instance");
    *inst = pimqap_instance{0, nullptr, nullptr};
    int32_t n = 0;
    pimqap_status st = pimqap_read_problem(path, PIMQAP_MAX_N, &n, nullptr, nullptr);
    if (st != PIMQAP_OK) return st;
    int32_t *F = static_cast<int32_t *>(std::malloc(sizeof(int32_t) * (size_t)n * n));
    int32_t *D = static_cast<int32_t *>(std::malloc(sizeof(int32_t) * (size_t)n * n));
    if (!F || !D) {
        std::free(F);
        std::free(D);
        return fail(PIMQAP_ERR_ARG, "out of host memory");
    }
    st = pimqap_read_problem(path, PIMQAP_MAX_N, &n, F, D);
    if (st != PIMQAP_OK) {
        std::free(F);
        std::free(D);
        return st;
    }
    *inst = pimqap_instance{n, F, D};
    return PIMQAP_OK;
}

void pimqap_free_instance(pimqap_instance *inst) {
    if (!inst) return;
    std::free(const_cast<int32_t *>(inst->flow));
    std::free(const_cast<int32_t *>(inst->dist));
    *inst = pimqap_instance{0, nullptr, nullptr};
}

pimqap_status pimqap_sweep_replay(const pimqap_instance *inst, const pimqap_params *params,
                                  const int32_t *phi_in, int32_t nsweeps, const double *r,
                                  int32_t *phi_out, int64_t *force, int64_t *energy,
                                  int64_t *best_energy, int64_t *accepts) {
    if (!inst || !params || !phi_in || !r || nsweeps < 0) return fail(PIMQAP_ERR_ARG, "bad replay arguments");
    if (params->update_rule != PIMQAP_RULE_SEQUENTIAL || params->active_facilities != 0)
        return fail(PIMQAP_ERR_ARG, "the replay runs CPU_PIM's sequential rule only");
    const int n = inst->n;
    if (n < 1 || n > PIMQAP_MAX_N) return fail(PIMQAP_ERR_ARG, "bad n");
    std::vector<char> seen((size_t)n, 0);
    for (int q = 0; q < n; ++q) {
        if (phi_in[q] < 0 || phi_in[q] >= n || seen[(size_t)phi_in[q]]) return fail(PIMQAP_ERR_ARG, "phi is not a permutation");
        seen[(size_t)phi_in[q]] = 1;
    }
    for (int64_t k = 0; k < (int64_t)nsweeps * n; ++k)
        if (!(r[k] >= 0.0 && r[k] < 1.0)) return fail(PIMQAP_ERR_ARG, "every r must be in [0, 1)");
    // one replica, one sweep per mega-iteration, no goal, no events: exactly nsweeps sweeps
    pimqap_params p = *params;
    p.replicas = 1;
    p.groups = 1;
    p.sweeps_per_exchange = 1;
    p.rank_slots = 0;
    p.auto_beta = 0;
    p.max_megaiters = nsweeps;
    p.goal = std::numeric_limits<int64_t>::min();
    p.timeout_s = 0;
    p.goal_print = 0;
    p.event_capacity = 0;
    pimqap_solver *s = nullptr;
    pimqap_status st = pimqap_solver_create(inst, &p, &s);
    if (st != PIMQAP_OK) return st;
    std::unique_ptr<pimqap_solver, void (*)(pimqap_solver *)> guard(s, pimqap_solver_destroy);
    double *dr = nullptr;
    struct FreeDev { void operator()(double *q) const { if (q) cudaFree(q); } };
    // the caller's permutation replaces the shuffle, then set-up runs again on it
    PQ_CUDA(cudaMemcpy(s->dev.phi, phi_in, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
    PQ_CUDA(pimqap::launch_setup(s->dev, s->bits, s->stream));
    if (nsweeps > 0) {
        PQ_CUDA(cudaMalloc(&dr, sizeof(double) * (size_t)nsweeps * n));
    }
    std::unique_ptr<double, FreeDev> rguard(dr);
    if (nsweeps > 0) {
        PQ_CUDA(cudaMemcpy(dr, r, sizeof(double) * (size_t)nsweeps * n, cudaMemcpyHostToDevice));
        s->dev.replay_r = dr;
        st = pimqap_solver_run(s, nsweeps, nullptr);
        if (st != PIMQAP_OK) return st;
    }
    PQ_CUDA(cudaStreamSynchronize(s->stream));
    st = pimqap_solver_replica(s, 0, 0, phi_out, force, energy, best_energy, nullptr);
    if (st != PIMQAP_OK) return st;
    if (accepts) {
        unsigned long long a = 0;
        PQ_CUDA(cudaMemcpy(&a, s->dev.accepts, 8, cudaMemcpyDeviceToHost));
        *accepts = (int64_t)a;
    }
    return PIMQAP_OK;
}

pimqap_status pimqap_solver_create(const pimqap_instance *inst, const pimqap_params *params,
                                   pimqap_solver **out) {
    if (!out) return fail(PIMQAP_ERR_ARG, "null output handle");
    *out = nullptr;
    pimqap_status st = check_params(inst, params);
    if (st != PIMQAP_OK) return st;
    auto s = new pimqap_solver();
    std::unique_ptr<pimqap_solver> guard(s);
    s->p = *params;
    s->device = params->device;
    int maxsm = 0;
    st = open_device(params->device, &maxsm);
    if (st != PIMQAP_OK) return st;
    Plan plan;
    st = plan_instance(inst, params, (size_t)maxsm, params->cluster_size, &plan);
    if (st != PIMQAP_OK) return st;
    st = plan_pairing(inst, params, (size_t)maxsm, &plan);
    if (st != PIMQAP_OK) return st;
    if (params->sweep_pipeline == 2) {   // the pipelined binary-flow epoch
        const size_t sp = pimqap::epoch_smem_bytes_pipe(plan.n, plan.rpc, plan.lds);
        if (!plan.bin || plan.act || plan.pair || params->launch_mode == 2 || sp > (size_t)maxsm)
            return fail(PIMQAP_ERR_ARG, "sweep_pipeline = 2 needs the binary-flow kernel (symmetric 0/1 flows, "
                                        "int16 distances, int32 forces), no clique moves, one replica per CTA "
                                        "set, launch_mode 0 or 1, and a layout that fits the cluster size");
        plan.pipe = true;
        plan.smem_bin = sp;
    }
    s->pipe = plan.pipe;
    s->pair = plan.pair;
    s->n = plan.n;
    s->T = plan.T;
    s->R = plan.R;
    s->cap = plan.cap;
    s->spe = plan.spe;
    s->sym = plan.sym;
    s->bin = plan.bin;
    s->bits = plan.bits;
    s->cl = plan.cl;
    s->threads = plan.threads;
    s->smem = plan.bin ? plan.smem_bin : plan.smem;
    PQ_CUDA(block_acquire(s->device, plan.total, &s->dmem, &s->dbytes));
    PQ_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    PQ_CUDA(cudaEventCreate(&s->ev0));
    PQ_CUDA(cudaEventCreate(&s->ev1));
    cudaStream_t q = s->stream;
    if (params->event_capacity > 0) {
        s->events.reset(new pimqap::detail::EventBuffer());
        const unsigned pcap = params->goal_print > 0
                                  ? (unsigned)(params->event_perm_capacity > 0 ? params->event_perm_capacity : 256)
                                  : 0u;
        // goalPrint acts only when positive (CPU_PIM.cpp:273)
        st = s->events->allocate((unsigned)params->event_capacity, pcap, plan.n,
                                 params->goal_print > 0 ? params->goal_print : 0, q);
        if (st != PIMQAP_OK) return st;
    }
    std::vector<std::vector<char>> keep;
    st = stage_instance(inst, params, plan, reinterpret_cast<char *>(s->dmem), &s->dev, q, keep,
                        s->events ? &s->events->link : nullptr);
    if (st != PIMQAP_OK) return st;
    SolveDev &d = s->dev;
    s->h2d = plan.h2d_bytes;
    s->beta0_used = params->beta_internal ? params->beta_max : params->beta_max * 1.44269504089;
    s->ratio_used = params->beta_ratio;
    PQ_CUDA(cudaStreamSynchronize(q));
    int32_t err = 0;
    PQ_CUDA(cudaMemcpy(&err, d.error, 4, cudaMemcpyDeviceToHost));
    s->d2h += 4;
    if (err) return fail(PIMQAP_ERR_DEVICE, "device check failed during setup");
    if (s->events) {
        PQ_CUDA(cudaMemcpy(&s->start_ns, d.start_ns, 8, cudaMemcpyDeviceToHost));
        st = s->events->drain(q, s->start_ns, true);
        if (st != PIMQAP_OK) return st;
    }
    // The whole run as one persistent launch per run call (launch_mode = 2) when every replica
    // can be resident at once.  Automatic mode keeps a CUDA graph of one launch per
    // mega-iteration: on the B200 its kernel boundaries cost no more than the persistent
    // launch's device barrier (n = 256, 64 replicas: 2.95e9 proposals/s both ways; n = 32,
    // 16 replicas, exchange every sweep: 1.60e8 against 1.49e8).  Solves with an event log keep
    // the graphs too: their log is drained between graph launches.
    if (params->launch_mode == 2 && s->pair)
        return fail(PIMQAP_ERR_ARG, "launch_mode = 2 needs every replica resident at once, no event log and "
                                    "one replica per CTA set");
    if (params->launch_mode == 2) {
        bool fits = false;
        PQ_CUDA(pimqap::solve_fits(d, s->bits, s->cl, s->sym, s->bin, s->threads, s->smem, &fits));
        const bool able = fits && !s->events;
        if (!able)
            return fail(PIMQAP_ERR_ARG, "launch_mode = 2 needs every replica resident at once, no event log and "
                                        "one replica per CTA set");
        if (able) {
            int32_t *k = nullptr;
            PQ_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&k), sizeof(int32_t), cudaHostAllocMapped));
            *k = 0;
            s->kill = k;
            int32_t *kd = nullptr;
            PQ_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void **>(&kd), k, 0));
            d.kill = kd;
            s->persistent = true;
        }
    }
    *out = guard.release();
    return PIMQAP_OK;
}

// pimqap_solver_run as one persistent launch: the launch runs mega-iterations up to
// run_end on the device; the host only waits, and on a timeout sets the kill word, which stops
// the launch at the next mega-iteration boundary.
static pimqap_status run_persistent(pimqap_solver *s, int64_t megaiters, double *device_ms) {
    const auto wall0 = std::chrono::steady_clock::now();
    int32_t done = 0;
    PQ_CUDA(cudaMemcpy(&done, s->dev.epoch_all, 4, cudaMemcpyDeviceToHost));
    s->d2h += 4;
    const int32_t end = (int32_t)std::min<int64_t>((int64_t)done + megaiters, (int64_t)pimqap::kNoStop - 1);
    double ms_total = 0;
    if (end > done && !s->stopped_goal) {
        if (!s->solve_graph) {
            cudaGraph_t graph;
            PQ_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = pimqap::launch_solve(s->dev, s->bits, s->cl, s->sym, s->bin, s->threads, s->smem,
                                                 s->stream);
            if (e != cudaSuccess) {
                cudaStreamEndCapture(s->stream, &graph);
                return fail(PIMQAP_ERR_CUDA, std::string("persistent launch: ") + cudaGetErrorString(e));
            }
            PQ_CUDA(cudaStreamEndCapture(s->stream, &graph));
            cudaError_t ie = cudaGraphInstantiate(&s->solve_graph, graph, 0);
            cudaGraphDestroy(graph);
            PQ_CUDA(ie);
        }
        *s->kill = 0;
        PQ_CUDA(cudaMemcpyAsync(const_cast<int32_t *>(s->dev.run_end), &end, 4, cudaMemcpyHostToDevice, s->stream));
        s->h2d += 4;
        PQ_CUDA(cudaEventRecord(s->ev0, s->stream));
        PQ_CUDA(cudaGraphLaunch(s->solve_graph, s->stream));
        ++s->launches;
        PQ_CUDA(cudaEventRecord(s->ev1, s->stream));
        if (s->p.timeout_s > 0) {
            // the -s stop (CPU_PIM.cpp:350-357): at the first boundary after the time is up
            for (;;) {
                const cudaError_t q = cudaEventQuery(s->ev1);
                if (q == cudaSuccess) break;
                if (q != cudaErrorNotReady) PQ_CUDA(q);
                const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
                if (el >= s->p.timeout_s) {
                    *s->kill = 1;
                    break;
                }
                std::this_thread::sleep_for(std::chrono::microseconds(200));
            }
        }
        PQ_CUDA(cudaStreamSynchronize(s->stream));
        float ms = 0;
        PQ_CUDA(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
        ms_total = ms;
    }
    int32_t epoch0 = 0, err = 0, stop = 0;
    PQ_CUDA(cudaMemcpy(&epoch0, s->dev.epoch, 4, cudaMemcpyDeviceToHost));
    PQ_CUDA(cudaMemcpy(&err, s->dev.error, 4, cudaMemcpyDeviceToHost));
    PQ_CUDA(cudaMemcpy(&stop, s->dev.stop_epoch, 4, cudaMemcpyDeviceToHost));
    s->d2h += 12;
    s->megaiters_done = epoch0;
    // a stop word set by the goal (not by the kill word) ends the solve for good
    if (stop != pimqap::kNoStop && !*s->kill) s->stopped_goal = true;
    if (*s->kill && stop != pimqap::kNoStop) {
        // the kill word moved the stop: clear it for a later run call unless the goal set it
        int64_t tepoch = 0;
        PQ_CUDA(cudaMemcpy(&tepoch, s->dev.target_epoch, 8, cudaMemcpyDeviceToHost));
        s->d2h += 8;
        if (tepoch != std::numeric_limits<int64_t>::max()) {
            s->stopped_goal = true;
        } else {
            const int32_t none = pimqap::kNoStop;
            PQ_CUDA(cudaMemcpy(s->dev.stop_epoch, &none, 4, cudaMemcpyHostToDevice));
            s->h2d += 4;
        }
    }
    s->device_ms += ms_total;
    if (device_ms) *device_ms = ms_total;
    if (err) return fail(PIMQAP_ERR_DEVICE, "device check failed (error word " + std::to_string(err) + ")");
    return PIMQAP_OK;
}

pimqap_status pimqap_solver_run(pimqap_solver *s, int64_t megaiters, double *device_ms) {
    if (!s) return fail(PIMQAP_ERR_ARG, "null solver");
    if (megaiters < 0) return fail(PIMQAP_ERR_ARG, "megaiters must be >= 0");
    PQ_CUDA(cudaSetDevice(s->device));
    if (s->persistent) return run_persistent(s, megaiters, device_ms);
    const auto wall0 = std::chrono::steady_clock::now();
    const int per = s->p.megaiters_per_launch > 0 ? s->p.megaiters_per_launch : 50;
    double ms_total = 0;
    int64_t left = megaiters;
    while (left > 0 && !s->stopped_goal) {
        const int g = (int)std::min<int64_t>(left, per);
        if (g != s->graph_epochs) {
            if (s->graph) {
                cudaGraphExecDestroy(s->graph);
                s->graph = nullptr;
            }
            cudaGraph_t graph;
            PQ_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
            for (int k = 0; k < g; ++k) {
                cudaError_t e = pimqap::launch_epoch(s->dev, s->bits, s->cl, s->sym, s->bin, s->threads,
                                                     s->smem, s->stream, s->pair, s->pipe);
                if (e != cudaSuccess) {
                    cudaStreamEndCapture(s->stream, &graph);
                    return fail(PIMQAP_ERR_CUDA, std::string("epoch launch: ") + cudaGetErrorString(e));
                }
            }
            PQ_CUDA(cudaStreamEndCapture(s->stream, &graph));
            cudaError_t ie = cudaGraphInstantiate(&s->graph, graph, 0);
            cudaGraphDestroy(graph);
            PQ_CUDA(ie);
            s->graph_epochs = g;
        }
        PQ_CUDA(cudaEventRecord(s->ev0, s->stream));
        PQ_CUDA(cudaGraphLaunch(s->graph, s->stream));
        s->launches += g;
        PQ_CUDA(cudaEventRecord(s->ev1, s->stream));
        int32_t stop = 0;
        PQ_CUDA(cudaMemcpyAsync(&stop, s->dev.stop_epoch, 4, cudaMemcpyDeviceToHost, s->stream));
        s->d2h += 4;
        PQ_CUDA(cudaStreamSynchronize(s->stream));
        float ms = 0;
        PQ_CUDA(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
        ms_total += ms;
        left -= g;
        if (stop != pimqap::kNoStop) s->stopped_goal = true;
        if (s->events) {
            pimqap_status est = s->events->drain(s->stream, s->start_ns, true);
            if (est != PIMQAP_OK) return est;
        }
        if (s->p.timeout_s > 0) {
            const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
            if (el >= s->p.timeout_s) break;
        }
    }
    int32_t epoch0 = 0, err = 0;
    PQ_CUDA(cudaMemcpy(&epoch0, s->dev.epoch, 4, cudaMemcpyDeviceToHost));
    PQ_CUDA(cudaMemcpy(&err, s->dev.error, 4, cudaMemcpyDeviceToHost));
    s->megaiters_done = epoch0;
    s->d2h += 8;
    s->device_ms += ms_total;
    if (device_ms) *device_ms = ms_total;
    if (err) return fail(PIMQAP_ERR_DEVICE, "device check failed (error word " + std::to_string(err) + ")");
    return PIMQAP_OK;
}

pimqap_status pimqap_solver_result(pimqap_solver *s, pimqap_result *r) {
    if (!s || !r) return fail(PIMQAP_ERR_ARG, "null solver or result");
    PQ_CUDA(cudaSetDevice(s->device));
    const size_t reps = (size_t)s->T * s->R;
    std::vector<int64_t> bestE(reps);
    std::vector<unsigned long long> acc(reps);
    int64_t single = 0, tepoch = 0;
    unsigned long long tns = 0, sns = 0;
    PQ_CUDA(cudaMemcpy(bestE.data(), s->dev.bestE, reps * 8, cudaMemcpyDeviceToHost));
    PQ_CUDA(cudaMemcpy(acc.data(), s->dev.accepts, reps * 8, cudaMemcpyDeviceToHost));
    PQ_CUDA(cudaMemcpy(&single, s->dev.single_best, 8, cudaMemcpyDeviceToHost));
    PQ_CUDA(cudaMemcpy(&tepoch, s->dev.target_epoch, 8, cudaMemcpyDeviceToHost));
    PQ_CUDA(cudaMemcpy(&tns, s->dev.target_ns, 8, cudaMemcpyDeviceToHost));
    PQ_CUDA(cudaMemcpy(&sns, s->dev.start_ns, 8, cudaMemcpyDeviceToHost));
    size_t arg = 0;
    for (size_t k = 1; k < reps; ++k)
        if (bestE[k] < bestE[arg]) arg = k;
    int32_t *perm_dst = r->best_perm;
    int64_t *energy_dst = r->final_energies;
    std::memset(r, 0, sizeof(*r));
    r->best_perm = perm_dst;
    r->final_energies = energy_dst;
    r->best_energy = std::min<int64_t>(bestE[arg], single);
    if (energy_dst) PQ_CUDA(cudaMemcpy(energy_dst, s->dev.E, reps * 8, cudaMemcpyDeviceToHost));
    r->beta_max_used = s->beta0_used;
    r->beta_ratio_used = s->ratio_used;
    if (perm_dst)
        PQ_CUDA(cudaMemcpy(perm_dst, s->dev.best_phi + arg * s->n, (size_t)s->n * 4, cudaMemcpyDeviceToHost));
    r->target_megaiter = (tepoch == std::numeric_limits<int64_t>::max()) ? -1 : tepoch;
    r->time_to_target_ms = (r->target_megaiter >= 0 && tns != ~0ull && tns >= sns) ? (double)(tns - sns) * 1e-6 : -1.0;
    r->megaiters_done = s->megaiters_done;
    r->updates = s->megaiters_done * (int64_t)s->spe * s->n * (int64_t)reps;
    r->sweeps = r->updates / s->n;
    r->proposals = r->sweeps * ((int64_t)s->n * (s->n - 1) / 2);
    int64_t a = 0;
    for (auto v : acc) a += (int64_t)v;
    r->accepts = a;
    r->device_ms = s->device_ms;
    r->force_bits = s->bits;
    r->cluster_size = s->cl;
    r->stopped_by = s->stopped_goal ? 1 : 0;
    r->launches = (int32_t)std::min<int64_t>(s->launches, 0x7fffffff);
    s->d2h += (int64_t)(reps * 16 + 8 * 4 + (perm_dst ? (size_t)s->n * 4 : 0));
    r->h2d_bytes = s->h2d;
    r->d2h_bytes = s->d2h;
    return PIMQAP_OK;
}

pimqap_status pimqap_solver_replica(pimqap_solver *s, int32_t t, int32_t l, int32_t *phi,
                                    int64_t *force, int64_t *energy, int64_t *best_energy,
                                    double *beta) {
    if (!s) return fail(PIMQAP_ERR_ARG, "null solver");
    if (t < 0 || t >= s->T || l < 0 || l >= s->R) return fail(PIMQAP_ERR_ARG, "replica index out of range");
    PQ_CUDA(cudaSetDevice(s->device));
    const size_t rep = (size_t)t * s->R + l;
    const int n = s->n;
    if (phi) PQ_CUDA(cudaMemcpy(phi, s->dev.phi + rep * n, (size_t)n * 4, cudaMemcpyDeviceToHost));
    if (energy) PQ_CUDA(cudaMemcpy(energy, s->dev.E + rep, 8, cudaMemcpyDeviceToHost));
    if (best_energy) PQ_CUDA(cudaMemcpy(best_energy, s->dev.bestE + rep, 8, cudaMemcpyDeviceToHost));
    if (beta) PQ_CUDA(cudaMemcpy(beta, s->dev.beta + rep, 8, cudaMemcpyDeviceToHost));
    if (force) {
        const int ld = s->dev.ldg;
        if (s->bits == 32) {
            std::vector<int32_t> tmp((size_t)n * ld);
            PQ_CUDA(cudaMemcpy(tmp.data(), reinterpret_cast<int32_t *>(s->dev.I) + rep * n * ld,
                               tmp.size() * 4, cudaMemcpyDeviceToHost));
            for (int i = 0; i < n; ++i)
                for (int a = 0; a < n; ++a) force[(size_t)i * n + a] = tmp[(size_t)i * ld + a];
        } else {
            std::vector<int64_t> tmp((size_t)n * ld);
            PQ_CUDA(cudaMemcpy(tmp.data(), reinterpret_cast<int64_t *>(s->dev.I) + rep * n * ld,
                               tmp.size() * 8, cudaMemcpyDeviceToHost));
            for (int i = 0; i < n; ++i)
                for (int a = 0; a < n; ++a) force[(size_t)i * n + a] = tmp[(size_t)i * ld + a];
        }
    }
    return PIMQAP_OK;
}

pimqap_status pimqap_solver_group(pimqap_solver *s, int32_t t, int32_t *order,
                                  int32_t *time_since_swap, int64_t *group_best) {
    if (!s) return fail(PIMQAP_ERR_ARG, "null solver");
    if (t < 0 || t >= s->T) return fail(PIMQAP_ERR_ARG, "group index out of range");
    PQ_CUDA(cudaSetDevice(s->device));
    if (order) PQ_CUDA(cudaMemcpy(order, s->dev.order + (size_t)t * s->cap, (size_t)s->cap * 4, cudaMemcpyDeviceToHost));
    if (time_since_swap) PQ_CUDA(cudaMemcpy(time_since_swap, s->dev.tss + t, 4, cudaMemcpyDeviceToHost));
    if (group_best) PQ_CUDA(cudaMemcpy(group_best, s->dev.group_best + t, 8, cudaMemcpyDeviceToHost));
    return PIMQAP_OK;
}

pimqap_status pimqap_solver_events(pimqap_solver *s, int64_t first, int32_t capacity,
                                   pimqap_event *events, int32_t *count, int64_t *total,
                                   int64_t *dropped) {
    if (!s || !count || capacity < 0 || first < 0 || (capacity > 0 && !events))
        return fail(PIMQAP_ERR_ARG, "bad event arguments");
    *count = 0;
    const int64_t have = s->events ? (int64_t)s->events->events.size() : 0;
    if (total) *total = have;
    if (dropped) *dropped = s->events ? s->events->dropped : 0;
    if (first >= have) return PIMQAP_OK;
    const int64_t k = std::min<int64_t>(capacity, have - first);
    std::memcpy(events, s->events->events.data() + first, sizeof(pimqap_event) * (size_t)k);
    *count = (int32_t)k;
    return PIMQAP_OK;
}

pimqap_status pimqap_solver_event_perm(pimqap_solver *s, int32_t perm_index, int32_t *perm) {
    if (!s || !perm) return fail(PIMQAP_ERR_ARG, "null solver or permutation");
    if (!s->events || perm_index < 0 || (size_t)perm_index * s->n >= s->events->perms.size())
        return fail(PIMQAP_ERR_ARG, "no permutation with that index");
    std::memcpy(perm, s->events->perms.data() + (size_t)perm_index * s->n, 4 * (size_t)s->n);
    return PIMQAP_OK;
}

void pimqap_solver_destroy(pimqap_solver *s) { delete s; }

pimqap_status pimqap_release_kept_memory(void) {
    KeptBlock take[kKeepDevices];
    {
        std::lock_guard<std::mutex> lk(g_keep_mu);
        for (int d = 0; d < kKeepDevices; ++d) {
            take[d] = g_keep[d];
            g_keep[d] = KeptBlock{};
        }
    }
    pimqap_status st = PIMQAP_OK;
    for (int d = 0; d < kKeepDevices; ++d) {
        if (!take[d].p) continue;
        const cudaError_t e = cudaFree(take[d].p);
        if (e != cudaSuccess && st == PIMQAP_OK)
            st = fail(PIMQAP_ERR_CUDA, std::string("cudaFree of a kept block: ") + cudaGetErrorString(e));
    }
    return st;
}

pimqap_status pimqap_solve(const pimqap_instance *inst, const pimqap_params *params,
                           pimqap_result *result) {
    if (!result) return fail(PIMQAP_ERR_ARG, "null result");
    if (!params) return fail(PIMQAP_ERR_ARG, "null params");
    const auto w0 = std::chrono::steady_clock::now();
    pimqap_params p = *params;
    int64_t auto_best = PIMQAP_NO_BEST;
    std::vector<int32_t> auto_perm;
    if (p.auto_beta) {   // automatic mode first (CPU_PIM.cpp:650-658)
        pimqap_status st = check_params(inst, params);
        if (st != PIMQAP_OK) return st;
        double b0 = 0, db = 0;
        auto_perm.assign(inst->n, 0);
        st = pimqap_auto_beta(inst, params, &b0, &db, nullptr, &auto_best, auto_perm.data());
        if (st != PIMQAP_OK) return st;
        p.auto_beta = 0;
        p.beta_internal = 1;
        p.beta_max = b0;
        p.beta_ratio = db;
        if (auto_best <= p.goal) p.max_megaiters = 0;   // the trials reached the goal (:420-422, :661)
    }
    pimqap_solver *s = nullptr;
    pimqap_status st = pimqap_solver_create(inst, &p, &s);
    if (st != PIMQAP_OK) return st;
    st = pimqap_solver_run(s, p.max_megaiters, nullptr);
    if (st == PIMQAP_OK) st = pimqap_solver_result(s, result);
    pimqap_solver_destroy(s);   // the handle's teardown is part of the call's wall time
    const double el = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
    if (st == PIMQAP_OK) {
        result->wall_ms = el;
        if (result->stopped_by == 0 && p.timeout_s > 0 && result->megaiters_done < p.max_megaiters)
            result->stopped_by = 2;
        if (auto_best < result->best_energy) {   // the trials' best counts (singleBestE carries over)
            result->best_energy = auto_best;
            if (result->best_perm) std::memcpy(result->best_perm, auto_perm.data(), 4 * (size_t)inst->n);
            if (auto_best <= p.goal) result->stopped_by = 1;
        }
    }
    return st;
}

}  // extern "C"
