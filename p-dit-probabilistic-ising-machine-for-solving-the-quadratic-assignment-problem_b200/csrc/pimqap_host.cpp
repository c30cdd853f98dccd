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
#include <cstring>
#include <fstream>
#include <limits>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "pimqap.h"
#include "pimqap_internal.h"

using pimqap::SolveDev;

namespace {

thread_local std::string g_error;

pimqap_status fail(pimqap_status st, const std::string &msg) {
    g_error = msg;
    return st;
}

}  // namespace

void pimqap::set_last_error(const char *msg) { g_error = msg; }

namespace {

#define PQ_CUDA(x)                                                                       \
    do {                                                                                 \
        cudaError_t e_ = (x);                                                            \
        if (e_ != cudaSuccess)                                                           \
            return fail(PIMQAP_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------------ random words (host)

// Philox4x32-10 (Salmon et al., SC'11).
void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = (uint32_t)p1;
        c[2] = n2;
        c[3] = (uint32_t)p0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// The shuffle stream as a C++ uniform random bit generator with the reference engine's
// interface (32-bit words, result_type uint_fast32_t), so std::uniform_int_distribution
// draws from it exactly as the reference's distN(rng[0]) draws from std::mt19937
// (CPU_PIM.cpp:147-148).  Word k is Philox({k/4, k>>34, 0, ~0}, seed)[k%4].
struct ShuffleEngine {
    typedef uint_fast32_t result_type;
    static constexpr result_type min() { return 0; }
    static constexpr result_type max() { return 0xFFFFFFFFu; }
    uint64_t seed = 0;
    uint64_t k = 0;
    result_type operator()() {
        uint32_t c[4] = {(uint32_t)(k >> 2), (uint32_t)(k >> 34), 0u, 0xFFFFFFFFu};
        philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
        return c[(k++) & 3];
    }
};

// Initial permutations of all groups (CPU_PIM.cpp:134-162): identity, then per group and
// location one draw j in [0, n) and the transposition (i j); all replicas of a group share it.
std::vector<int32_t> initial_perms(int n, int T, uint64_t seed) {
    std::vector<int32_t> perms((size_t)T * n);
    ShuffleEngine eng;
    eng.seed = seed;
    for (int t = 0; t < T; ++t) {
        int32_t *p = perms.data() + (size_t)t * n;
        for (int i = 0; i < n; ++i) p[i] = i;
        for (int i = 0; i < n; ++i) {
            std::uniform_int_distribution<ShuffleEngine::result_type> distN(0, n - 1);
            const int j = (int)distN(eng);
            if (i != j) std::swap(p[i], p[j]);
        }
    }
    return perms;
}

// ------------------------------------------------------------------ instance analysis

struct InstanceInfo {
    bool symmetric = false;
    int bits_needed = 32;   // 32, 64, or 0 when even int64 is not provably safe
};

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

}  // namespace

// ------------------------------------------------------------------ solver object

struct pimqap_solver {
    pimqap_params p{};
    int n = 0, T = 0, R = 0, cap = 0, spe = 0;
    int bits = 32, cl = 1, threads = 256;
    bool sym = false;
    size_t smem = 0;
    int device = 0;
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

    ~pimqap_solver() {
        if (graph) cudaGraphExecDestroy(graph);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
        if (dmem) cudaFree(dmem);
    }
};

namespace {

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
    if (p->force_bits != 0 && p->force_bits != 32 && p->force_bits != 64)
        return fail(PIMQAP_ERR_ARG, "force_bits must be 0, 32 or 64");
    if (p->threads_per_block != 0 && p->threads_per_block != 64 && p->threads_per_block != 128 &&
        p->threads_per_block != 256)
        return fail(PIMQAP_ERR_ARG, "threads_per_block must be 0, 64, 128 or 256");
    if (p->cluster_size != 0 && p->cluster_size != 1 && p->cluster_size != 2 && p->cluster_size != 4)
        return fail(PIMQAP_ERR_ARG, "cluster_size must be 0, 1, 2 or 4");
    return PIMQAP_OK;
}

template <class T> T *carve(char *&cur, size_t count) {
    T *p = reinterpret_cast<T *>(cur);
    cur += (count * sizeof(T) + 255) & ~size_t(255);
    return p;
}

size_t carve_size(size_t bytes) { return (bytes + 255) & ~size_t(255); }

// ------------------------------------------------------------------ per-instance plan + staging

// Everything decided for one instance before device memory is touched.
struct Plan {
    int n = 0, T = 0, R = 0, cap = 0, spe = 0;
    int bits = 32, cl = 1, threads = 256;
    int npad = 0, lds = 0, ldm = 0, rpc = 0;
    bool sym = false;
    size_t smem = 0;       // epoch kernel shared memory per CTA
    size_t total = 0;      // device bytes of the instance's SolveDev arrays
    int64_t h2d_bytes = 0;
};

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

// Force-matrix width, symmetry, launch shape (threads, the smallest cluster whose row share of
// I fits one CTA, or `want_cluster`), strides and the device footprint.
pimqap_status plan_instance(const pimqap_instance *inst, const pimqap_params *params, size_t maxsm,
                            int want_cluster, Plan *out) {
    const int n = inst->n;
    const InstanceInfo info = analyse(n, inst->flow, inst->dist);
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
    const size_t reps = (size_t)P.T * P.R, nn = (size_t)n * P.ldm;
    P.total = carve_size(reps * (size_t)n * P.npad * isz) + 4 * carve_size(nn * 4) +
              2 * carve_size((size_t)n * 4) + 2 * carve_size(reps * n * 4) + 4 * carve_size(reps * 8) +
              carve_size((size_t)P.T * P.cap * 4) + 4 * carve_size((size_t)P.T * 8) + 8 * carve_size(8);
    P.h2d_bytes = (int64_t)(4 * nn * 4 + 2 * (size_t)n * 4 + reps * n * 4 + reps * 8 +
                            (size_t)P.T * P.cap * 4 + (size_t)P.T * 8 + 8 + 4 + 8 + 8);
    *out = P;
    return PIMQAP_OK;
}

// setup() for one instance (CPU_PIM.cpp:109-193): carves the SolveDev arrays out of `base`
// (plan.total bytes), uploads the padded matrices, transposes, diagonals, initial
// permutations, beta ladder and rank slots on stream q, and enqueues the setup kernels.  The
// host buffers of the asynchronous copies are kept in `keep` until the caller syncs q.
pimqap_status stage_instance(const pimqap_instance *inst, const pimqap_params *params,
                             const Plan &P, char *base, SolveDev *out, cudaStream_t q,
                             std::vector<std::vector<char>> &keep) {
    const int n = P.n, T = P.T, R = P.R, cap = P.cap, ldm = P.ldm;
    const size_t reps = (size_t)T * R, nn = (size_t)n * ldm;
    auto buffer = [&](size_t bytes) -> char * {
        keep.emplace_back(bytes, 0);
        return keep.back().data();
    };
    int32_t *Dp = reinterpret_cast<int32_t *>(buffer(nn * 4));
    int32_t *DT = reinterpret_cast<int32_t *>(buffer(nn * 4));
    int32_t *Fp = reinterpret_cast<int32_t *>(buffer(nn * 4));
    int32_t *FT = reinterpret_cast<int32_t *>(buffer(nn * 4));
    int32_t *Dd = reinterpret_cast<int32_t *>(buffer((size_t)n * 4));
    int32_t *Fd = reinterpret_cast<int32_t *>(buffer((size_t)n * 4));
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
    int32_t *phi = reinterpret_cast<int32_t *>(buffer(reps * n * 4));
    for (int t = 0; t < T; ++t)
        for (int l = 0; l < R; ++l)
            std::memcpy(&phi[((size_t)t * R + l) * n], &perms[(size_t)t * n], sizeof(int32_t) * n);
    // beta ladder (CPU_PIM.cpp:111-119); -b is given in natural units and stored x 1/ln 2 (:528)
    const double beta0 = params->beta_max * 1.44269504089;
    double *beta = reinterpret_cast<double *>(buffer(reps * 8));
    for (int t = 0; t < T; ++t) {
        double running = beta0;
        for (int l = R - 1; l >= 0; --l) {
            beta[(size_t)t * R + l] = running;
            running /= params->beta_ratio;
        }
    }
    int32_t *order = reinterpret_cast<int32_t *>(buffer((size_t)T * cap * 4));
    for (int t = 0; t < T; ++t)
        for (int l = 0; l < R; ++l) order[(size_t)t * cap + l] = l;
    int64_t *nob = reinterpret_cast<int64_t *>(buffer((size_t)(T + 1) * 8));
    for (int t = 0; t <= T; ++t) nob[t] = pimqap::kNoBest;
    int64_t *consts = reinterpret_cast<int64_t *>(buffer(3 * 8));
    consts[0] = pimqap::kNoStop;
    consts[1] = std::numeric_limits<int64_t>::max();
    consts[2] = (int64_t)~0ull;

    PQ_CUDA(cudaMemsetAsync(base, 0, P.total, q));
    char *cur = base;
    SolveDev d{};
    d.n = n; d.R = R; d.T = T; d.cap = cap; d.spe = P.spe;
    d.ldg = P.npad; d.lds = P.lds; d.ldm = ldm; d.rpc = P.rpc;
    d.goal = params->goal;
    d.seed = params->seed;
    d.I = carve<char>(cur, reps * (size_t)n * P.npad * (P.bits / 8));
    int32_t *dD = carve<int32_t>(cur, nn), *dDT = carve<int32_t>(cur, nn);
    int32_t *dF = carve<int32_t>(cur, nn), *dFT = carve<int32_t>(cur, nn);
    int32_t *dDd = carve<int32_t>(cur, n), *dFd = carve<int32_t>(cur, n);
    d.D = dD; d.DT = dDT; d.F = dF; d.FT = dFT; d.Ddiag = dDd; d.Fdiag = dFd;
    d.phi = carve<int32_t>(cur, reps * n);
    d.best_phi = carve<int32_t>(cur, reps * n);
    d.E = carve<int64_t>(cur, reps);
    d.bestE = carve<int64_t>(cur, reps);
    d.beta = carve<double>(cur, reps);
    d.accepts = carve<unsigned long long>(cur, reps);
    d.order = carve<int32_t>(cur, (size_t)T * cap);
    d.tss = carve<int32_t>(cur, T);
    d.group_best = carve<int64_t>(cur, T);
    d.finish = carve<unsigned int>(cur, T);
    d.epoch = carve<int32_t>(cur, T);
    d.single_best = carve<int64_t>(cur, 1);
    d.stop_epoch = carve<int32_t>(cur, 1);
    d.target_epoch = carve<int64_t>(cur, 1);
    d.target_ns = carve<unsigned long long>(cur, 1);
    d.start_ns = carve<unsigned long long>(cur, 1);
    d.error = carve<int32_t>(cur, 1);
    if ((size_t)(cur - base) > P.total) return fail(PIMQAP_ERR_ARG, "internal: device carve overflow");
    PQ_CUDA(cudaMemcpyAsync(dD, Dp, nn * 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(dF, Fp, nn * 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(dDT, DT, nn * 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(dFT, FT, nn * 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(dDd, Dd, (size_t)n * 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(dFd, Fd, (size_t)n * 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d.phi, phi, reps * n * 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d.beta, beta, reps * 8, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d.order, order, (size_t)T * cap * 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d.group_best, nob, (size_t)T * 8, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d.single_best, nob + T, 8, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d.stop_epoch, &consts[0], 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d.target_epoch, &consts[1], 8, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d.target_ns, &consts[2], 8, cudaMemcpyHostToDevice, q));
    PQ_CUDA(pimqap::launch_setup(d, P.bits, q));
    *out = d;
    return PIMQAP_OK;
}

// Worker shape of a persistent class (the autotuner's knobs): threads per replica worker,
// workers per CTA (named barriers 1..8) and the shared-memory slice of one worker.
struct BatchShape {
    int worker_threads = 128, workers = 1, ctas_per_sm = 1, grid = 1;
    size_t slice = 0;
};

BatchShape batch_shape(const std::vector<Plan> &plans, const std::vector<int> &members, int bits,
                       int sms, int maxsm) {
    BatchShape S;
    int nmax = 0;
    for (int k : members) {
        S.slice = std::max(S.slice, pimqap::batch_slice_bytes(plans[k].n, bits));
        nmax = std::max(nmax, plans[k].n);
    }
    S.worker_threads = nmax <= 32 ? 32 : (nmax <= 64 ? 64 : 128);
    S.workers = std::max(1, std::min(256 / S.worker_threads, (int)((size_t)maxsm / S.slice)));
    int occ = 0;
    if (pimqap::batch_occupancy(bits, S.workers * S.worker_threads, S.workers * S.slice, &occ) != cudaSuccess || occ < 1)
        occ = 1;
    S.ctas_per_sm = occ;
    S.grid = sms * occ;
    return S;
}

// Solves `members` (single-CTA replicas of one force-matrix width) in one persistent launch.
pimqap_status run_batch_class(const pimqap_instance *insts, const pimqap_params *params,
                              const std::vector<Plan> &plans, const std::vector<int> &members,
                              int bits, int sms, int maxsm, pimqap_result *results) {
    const int m = (int)members.size();
    const BatchShape S = batch_shape(plans, members, bits, sms, maxsm);
    size_t reps_total = 0, inst_bytes = 0;
    std::vector<size_t> offs(m);
    for (int q = 0; q < m; ++q) {
        const Plan &P = plans[members[q]];
        offs[q] = inst_bytes;
        inst_bytes += carve_size(P.total);
        reps_total += (size_t)P.T * P.R;
    }
    unsigned qcap = 1;
    while (qcap < reps_total + 1) qcap <<= 1;
    const size_t total = inst_bytes + carve_size(sizeof(SolveDev) * m) + 3 * carve_size(8 * (size_t)m) +
                         2 * carve_size(8 * (size_t)qcap) + 6 * carve_size(8);
    char *base = nullptr;
    PQ_CUDA(cudaMalloc(&base, total));
    struct Free {
        char *p;
        ~Free() { cudaFree(p); }
    } free_guard{base};
    cudaStream_t q = nullptr;
    PQ_CUDA(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
    struct FreeStream {
        cudaStream_t s;
        ~FreeStream() { cudaStreamDestroy(s); }
    } stream_guard{q};

    std::vector<SolveDev> devs(m);
    std::vector<std::vector<char>> keep;
    for (int i = 0; i < m; ++i) {
        const int k = members[i];
        pimqap_status st = stage_instance(&insts[k], &params[k], plans[k], base + offs[i], &devs[i], q, keep);
        if (st != PIMQAP_OK) return st;
    }
    char *cur = base + inst_bytes;
    SolveDev *d_inst = carve<SolveDev>(cur, m);
    int32_t *d_sym = reinterpret_cast<int32_t *>(carve<int64_t>(cur, m));
    int64_t *d_maxm = carve<int64_t>(cur, m);
    unsigned int *d_finish = reinterpret_cast<unsigned int *>(carve<int64_t>(cur, m));
    unsigned long long *d_items = carve<unsigned long long>(cur, qcap);
    unsigned long long *d_seq = carve<unsigned long long>(cur, qcap);
    unsigned long long *d_head = carve<unsigned long long>(cur, 1);
    unsigned long long *d_tail = carve<unsigned long long>(cur, 1);
    int32_t *d_active = reinterpret_cast<int32_t *>(carve<int64_t>(cur, 1));
    int32_t *d_error = reinterpret_cast<int32_t *>(carve<int64_t>(cur, 1));
    unsigned long long *d_start = carve<unsigned long long>(cur, 1);
    PQ_CUDA(cudaMemsetAsync(base + inst_bytes, 0, total - inst_bytes, q));

    PQ_CUDA(cudaStreamSynchronize(q));
    keep.clear();
    std::vector<int32_t> stop0(m);
    for (int i = 0; i < m; ++i)
        PQ_CUDA(cudaMemcpy(&stop0[i], devs[i].stop_epoch, 4, cudaMemcpyDeviceToHost));
    // Epoch-0 items, largest instances first (they take longest).
    std::vector<int> order_idx(m);
    for (int i = 0; i < m; ++i) order_idx[i] = i;
    std::stable_sort(order_idx.begin(), order_idx.end(), [&](int a, int b) {
        const Plan &A = plans[members[a]], &B = plans[members[b]];
        return (double)A.n * A.n * A.T * A.R > (double)B.n * B.n * B.T * B.R;
    });
    std::vector<int32_t> sym(2 * m, 0);
    std::vector<int64_t> maxm(m);
    std::vector<unsigned long long> items, seq;
    int active = 0;
    for (int i = 0; i < m; ++i) {
        sym[i] = plans[members[i]].sym ? 1 : 0;
        maxm[i] = params[members[i]].max_megaiters;
    }
    for (int i : order_idx) {
        const Plan &P = plans[members[i]];
        if (maxm[i] <= 0 || stop0[i] <= 0) continue;   // nothing to run, or goal met at setup
        ++active;
        for (int r = 0; r < P.T * P.R; ++r) {
            items.push_back(((unsigned long long)i << 32) | (unsigned)r);
            seq.push_back(items.size());
        }
    }
    const unsigned long long tail = items.size();
    PQ_CUDA(cudaMemcpyAsync(d_inst, devs.data(), sizeof(SolveDev) * m, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d_sym, sym.data(), 4 * (size_t)m, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d_maxm, maxm.data(), 8 * (size_t)m, cudaMemcpyHostToDevice, q));
    if (!items.empty()) {
        PQ_CUDA(cudaMemcpyAsync(d_items, items.data(), 8 * items.size(), cudaMemcpyHostToDevice, q));
        PQ_CUDA(cudaMemcpyAsync(d_seq, seq.data(), 8 * seq.size(), cudaMemcpyHostToDevice, q));
    }
    PQ_CUDA(cudaMemcpyAsync(d_tail, &tail, 8, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d_active, &active, 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaStreamSynchronize(q));
    keep.clear();

    pimqap::BatchDev B{};
    B.inst = d_inst; B.sym = d_sym; B.max_megaiters = d_maxm; B.finish_inst = d_finish;
    B.count = m; B.q_items = d_items; B.q_seq = d_seq; B.q_head = d_head; B.q_tail = d_tail;
    B.qmask = qcap - 1; B.active = d_active; B.error = d_error; B.start_ns = d_start;
    B.worker_threads = S.worker_threads; B.workers = S.workers; B.slice_bytes = (unsigned)S.slice;
    cudaEvent_t e0, e1;
    PQ_CUDA(cudaEventCreate(&e0));
    PQ_CUDA(cudaEventCreate(&e1));
    PQ_CUDA(cudaEventRecord(e0, q));
    if (active > 0) PQ_CUDA(pimqap::launch_batch(B, bits, S.grid, q));
    PQ_CUDA(cudaEventRecord(e1, q));
    PQ_CUDA(cudaStreamSynchronize(q));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int32_t err = 0;
    unsigned long long start_ns = 0;
    PQ_CUDA(cudaMemcpy(&err, d_error, 4, cudaMemcpyDeviceToHost));
    PQ_CUDA(cudaMemcpy(&start_ns, d_start, 8, cudaMemcpyDeviceToHost));
    if (err) return fail(PIMQAP_ERR_DEVICE, "batch kernel check failed (error word " + std::to_string(err) + ")");

    for (int i = 0; i < m; ++i) {
        const int k = members[i];
        const SolveDev &d = devs[i];
        const Plan &P = plans[k];
        const size_t reps = (size_t)P.T * P.R;
        std::vector<int64_t> bestE(reps);
        std::vector<unsigned long long> acc(reps);
        int64_t single = 0, tepoch = 0;
        unsigned long long tns = 0;
        int32_t epoch0 = 0, ierr = 0;
        PQ_CUDA(cudaMemcpy(bestE.data(), d.bestE, reps * 8, cudaMemcpyDeviceToHost));
        PQ_CUDA(cudaMemcpy(acc.data(), d.accepts, reps * 8, cudaMemcpyDeviceToHost));
        PQ_CUDA(cudaMemcpy(&single, d.single_best, 8, cudaMemcpyDeviceToHost));
        PQ_CUDA(cudaMemcpy(&tepoch, d.target_epoch, 8, cudaMemcpyDeviceToHost));
        PQ_CUDA(cudaMemcpy(&tns, d.target_ns, 8, cudaMemcpyDeviceToHost));
        PQ_CUDA(cudaMemcpy(&epoch0, d.epoch, 4, cudaMemcpyDeviceToHost));
        PQ_CUDA(cudaMemcpy(&ierr, d.error, 4, cudaMemcpyDeviceToHost));
        if (ierr) return fail(PIMQAP_ERR_DEVICE, "device check failed in batch instance " + std::to_string(k));
        size_t arg = 0;
        for (size_t r = 1; r < reps; ++r)
            if (bestE[r] < bestE[arg]) arg = r;
        pimqap_result &R = results[k];
        int32_t *perm_dst = R.best_perm;
        std::memset(&R, 0, sizeof(R));
        R.best_perm = perm_dst;
        R.best_energy = std::min<int64_t>(bestE[arg], single);
        if (perm_dst)
            PQ_CUDA(cudaMemcpy(perm_dst, d.best_phi + arg * P.n, (size_t)P.n * 4, cudaMemcpyDeviceToHost));
        R.target_megaiter = (tepoch == std::numeric_limits<int64_t>::max()) ? -1 : tepoch;
        R.time_to_target_ms = (R.target_megaiter >= 0 && tns != ~0ull && tns >= start_ns)
                                  ? (double)(tns - start_ns) * 1e-6 : (R.target_megaiter >= 0 ? 0.0 : -1.0);
        R.megaiters_done = epoch0;
        R.updates = (int64_t)epoch0 * P.spe * P.n * (int64_t)reps;
        int64_t a = 0;
        for (auto v : acc) a += (int64_t)v;
        R.accepts = a;
        R.device_ms = ms;
        R.force_bits = P.bits;
        R.cluster_size = 1;
        int32_t stop = 0;
        PQ_CUDA(cudaMemcpy(&stop, d.stop_epoch, 4, cudaMemcpyDeviceToHost));
        R.stopped_by = (stop != pimqap::kNoStop) ? 1 : 0;
        R.h2d_bytes = P.h2d_bytes;
        R.d2h_bytes = (int64_t)(reps * 16 + 40 + (perm_dst ? (size_t)P.n * 4 : 0));
    }
    return PIMQAP_OK;
}

}  // namespace

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
    s->n = plan.n;
    s->T = plan.T;
    s->R = plan.R;
    s->cap = plan.cap;
    s->spe = plan.spe;
    s->sym = plan.sym;
    s->bits = plan.bits;
    s->cl = plan.cl;
    s->threads = plan.threads;
    s->smem = plan.smem;
    PQ_CUDA(cudaMalloc(&s->dmem, plan.total));
    s->dbytes = plan.total;
    PQ_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    PQ_CUDA(cudaEventCreate(&s->ev0));
    PQ_CUDA(cudaEventCreate(&s->ev1));
    cudaStream_t q = s->stream;
    std::vector<std::vector<char>> keep;
    st = stage_instance(inst, params, plan, reinterpret_cast<char *>(s->dmem), &s->dev, q, keep);
    if (st != PIMQAP_OK) return st;
    SolveDev &d = s->dev;
    s->h2d = plan.h2d_bytes;
    PQ_CUDA(cudaStreamSynchronize(q));
    int32_t err = 0;
    PQ_CUDA(cudaMemcpy(&err, d.error, 4, cudaMemcpyDeviceToHost));
    s->d2h += 4;
    if (err) return fail(PIMQAP_ERR_DEVICE, "device check failed during setup");
    *out = guard.release();
    return PIMQAP_OK;
}

pimqap_status pimqap_solver_run(pimqap_solver *s, int64_t megaiters, double *device_ms) {
    if (!s) return fail(PIMQAP_ERR_ARG, "null solver");
    if (megaiters < 0) return fail(PIMQAP_ERR_ARG, "megaiters must be >= 0");
    PQ_CUDA(cudaSetDevice(s->device));
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
                cudaError_t e = pimqap::launch_epoch(s->dev, s->bits, s->cl, s->sym, s->threads,
                                                     s->smem, s->stream);
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
    std::memset(r, 0, sizeof(*r));
    r->best_perm = perm_dst;
    r->best_energy = std::min<int64_t>(bestE[arg], single);
    if (perm_dst)
        PQ_CUDA(cudaMemcpy(perm_dst, s->dev.best_phi + arg * s->n, (size_t)s->n * 4, cudaMemcpyDeviceToHost));
    r->target_megaiter = (tepoch == std::numeric_limits<int64_t>::max()) ? -1 : tepoch;
    r->time_to_target_ms = (r->target_megaiter >= 0 && tns != ~0ull && tns >= sns) ? (double)(tns - sns) * 1e-6 : -1.0;
    r->megaiters_done = s->megaiters_done;
    r->updates = s->megaiters_done * (int64_t)s->spe * s->n * (int64_t)reps;
    int64_t a = 0;
    for (auto v : acc) a += (int64_t)v;
    r->accepts = a;
    r->device_ms = s->device_ms;
    r->force_bits = s->bits;
    r->cluster_size = s->cl;
    r->stopped_by = s->stopped_goal ? 1 : 0;
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

void pimqap_solver_destroy(pimqap_solver *s) { delete s; }

pimqap_status pimqap_solve(const pimqap_instance *inst, const pimqap_params *params,
                           pimqap_result *result) {
    if (!result) return fail(PIMQAP_ERR_ARG, "null result");
    const auto w0 = std::chrono::steady_clock::now();
    pimqap_solver *s = nullptr;
    pimqap_status st = pimqap_solver_create(inst, params, &s);
    if (st != PIMQAP_OK) return st;
    st = pimqap_solver_run(s, params->max_megaiters, nullptr);
    if (st == PIMQAP_OK) st = pimqap_solver_result(s, result);
    const double el = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
    if (st == PIMQAP_OK) {
        result->wall_ms = el;
        if (result->stopped_by == 0 && params->timeout_s > 0 && result->megaiters_done < params->max_megaiters)
            result->stopped_by = 2;
    }
    pimqap_solver_destroy(s);
    return st;
}

pimqap_status pimqap_batch_solve(const pimqap_instance *insts, const pimqap_params *params,
                                 int32_t count, pimqap_result *results) {
    if (count < 0 || (count > 0 && (!insts || !params || !results)))
        return fail(PIMQAP_ERR_ARG, "bad batch arguments");
    if (count == 0) return PIMQAP_OK;
    const auto wall0 = std::chrono::steady_clock::now();
    for (int k = 0; k < count; ++k) {
        pimqap_status st = check_params(&insts[k], &params[k]);
        if (st != PIMQAP_OK) return st;
        if (params[k].device != params[0].device)
            return fail(PIMQAP_ERR_ARG, "every batch entry must use the same device");
    }
    int maxsm = 0;
    pimqap_status st = open_device(params[0].device, &maxsm);
    if (st != PIMQAP_OK) return st;
    int sms = 0;
    PQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, params[0].device));

    std::vector<Plan> plans(count);
    for (int k = 0; k < count; ++k) {
        st = plan_instance(&insts[k], &params[k], (size_t)maxsm, params[k].cluster_size, &plans[k]);
        if (st != PIMQAP_OK) return st;
    }
    // Persistent classes: single-CTA replicas by force-matrix width.  Replicas that need a
    // cluster are solved by the epoch launches of pimqap_solve.
    std::vector<int> cluster_members;
    for (int bits : {32, 64}) {
        std::vector<int> members;
        for (int k = 0; k < count; ++k) {
            if (plans[k].bits != bits) continue;
            if (plans[k].cl != 1 || pimqap::batch_slice_bytes(plans[k].n, bits) > (size_t)maxsm) continue;
            members.push_back(k);
        }
        if (members.empty()) continue;
        st = run_batch_class(insts, params, plans, members, bits, sms, maxsm, results);
        if (st != PIMQAP_OK) return st;
    }
    for (int k = 0; k < count; ++k) {
        const bool in_class = plans[k].cl == 1 &&
                              pimqap::batch_slice_bytes(plans[k].n, plans[k].bits) <= (size_t)maxsm;
        if (in_class) continue;
        st = pimqap_solve(&insts[k], &params[k], &results[k]);
        if (st != PIMQAP_OK) return st;
    }
    const double el = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall0).count();
    for (int k = 0; k < count; ++k) results[k].wall_ms = el;
    return PIMQAP_OK;
}

}  // extern "C"
