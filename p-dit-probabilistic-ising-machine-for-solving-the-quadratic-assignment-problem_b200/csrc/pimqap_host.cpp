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
    return PIMQAP_OK;
}

template <class T> T *carve(char *&cur, size_t count) {
    T *p = reinterpret_cast<T *>(cur);
    cur += (count * sizeof(T) + 255) & ~size_t(255);
    return p;
}

size_t carve_size(size_t bytes) { return (bytes + 255) & ~size_t(255); }

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
    const int n = inst->n;
    const InstanceInfo info = analyse(n, inst->flow, inst->dist);
    if (info.bits_needed == 0 && params->force_bits == 0)
        return fail(PIMQAP_ERR_RANGE, "instance values can overflow int64 force matrices");

    auto s = new pimqap_solver();
    std::unique_ptr<pimqap_solver> guard(s);
    s->p = *params;
    s->n = n;
    s->T = params->groups;
    s->R = params->replicas;
    s->cap = params->rank_slots ? params->rank_slots : std::max(params->replicas, 10);
    s->spe = params->sweeps_per_exchange;
    s->sym = info.symmetric;
    s->bits = params->force_bits ? params->force_bits : info.bits_needed;
    s->device = params->device;

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(PIMQAP_ERR_NO_DEVICE, "no CUDA device");
    if (s->device < 0 || s->device >= ndev) return fail(PIMQAP_ERR_ARG, "bad device ordinal");
    PQ_CUDA(cudaSetDevice(s->device));
    cudaDeviceProp prop;
    PQ_CUDA(cudaGetDeviceProperties(&prop, s->device));
    if (prop.major != 10) return fail(PIMQAP_ERR_NO_DEVICE, "the kernels are built for sm_100a only");
    PQ_CUDA(pimqap::prepare_kernels());

    // Launch shape: threads per CTA and the smallest cluster whose row share fits.
    const int isz = s->bits / 8, vec = 16 / isz;
    const int npad = round_up(n, 4);
    int lds = npad;
    if ((lds / vec) % 2 == 0) lds += vec;
    s->threads = params->threads_per_block ? params->threads_per_block
                                           : (n <= 64 ? 64 : (n <= 128 ? 128 : 256));
    const size_t maxsm = prop.sharedMemPerBlockOptin;
    s->cl = 0;
    for (int cl : {1, 2, 4}) {
        const int rpc = (n + cl - 1) / cl;
        if (pimqap::epoch_smem_bytes(n, rpc, lds, cl, s->bits) <= maxsm) {
            s->cl = cl;
            break;
        }
    }
    if (!s->cl) return fail(PIMQAP_ERR_ARG, "force matrix does not fit a 4-CTA cluster");
    const int rpc = (n + s->cl - 1) / s->cl;
    s->smem = pimqap::epoch_smem_bytes(n, rpc, lds, s->cl, s->bits);

    // Host-side setup: transposes, diagonals, permutations, beta ladder, rank slots.
    const int T = s->T, R = s->R, cap = s->cap;
    const size_t reps = (size_t)T * R, nn = (size_t)n * n;
    std::vector<int32_t> DT(nn), FT(nn), Dd(n), Fd(n);
    for (int i = 0; i < n; ++i) {
        Dd[i] = inst->dist[i * n + i];
        Fd[i] = inst->flow[i * n + i];
        for (int j = 0; j < n; ++j) {
            DT[i * n + j] = inst->dist[j * n + i];
            FT[i * n + j] = inst->flow[j * n + i];
        }
    }
    const std::vector<int32_t> perms = initial_perms(n, T, params->seed);
    std::vector<int32_t> phi(reps * n);
    for (int t = 0; t < T; ++t)
        for (int l = 0; l < R; ++l)
            std::memcpy(&phi[((size_t)t * R + l) * n], &perms[(size_t)t * n], sizeof(int32_t) * n);
    // beta ladder (CPU_PIM.cpp:111-119); -b is given in natural units and stored x 1/ln 2 (:528)
    const double beta0 = params->beta_max * 1.44269504089;
    std::vector<double> beta(reps);
    for (int t = 0; t < T; ++t) {
        double running = beta0;
        for (int l = R - 1; l >= 0; --l) {
            beta[(size_t)t * R + l] = running;
            running /= params->beta_ratio;
        }
    }
    std::vector<int32_t> order((size_t)T * cap, 0);
    for (int t = 0; t < T; ++t)
        for (int l = 0; l < R; ++l) order[(size_t)t * cap + l] = l;

    // Device memory: one allocation carved into the arrays of SolveDev.
    const size_t Ibytes = reps * (size_t)n * npad * isz;
    size_t total = carve_size(Ibytes) + 4 * carve_size(nn * 4) + 2 * carve_size(n * 4) +
                   2 * carve_size(reps * n * 4) + 4 * carve_size(reps * 8) +
                   carve_size((size_t)T * cap * 4) + 4 * carve_size((size_t)T * 8) +
                   8 * carve_size(8);
    PQ_CUDA(cudaMalloc(&s->dmem, total));
    s->dbytes = total;
    PQ_CUDA(cudaMemset(s->dmem, 0, total));
    char *cur = reinterpret_cast<char *>(s->dmem);
    SolveDev &d = s->dev;
    d.n = n; d.R = R; d.T = T; d.cap = cap; d.spe = s->spe;
    d.ldg = npad; d.lds = lds; d.rpc = rpc;
    d.goal = params->goal;
    d.seed = params->seed;
    d.I = carve<char>(cur, Ibytes);
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
    if ((size_t)(cur - reinterpret_cast<char *>(s->dmem)) > total)
        return fail(PIMQAP_ERR_ARG, "internal: device carve overflow");

    PQ_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    PQ_CUDA(cudaEventCreate(&s->ev0));
    PQ_CUDA(cudaEventCreate(&s->ev1));
    cudaStream_t q = s->stream;
    s->h2d = (int64_t)(4 * nn * 4 + 2 * (size_t)n * 4 + reps * n * 4 + reps * 8 + (size_t)T * cap * 4 +
                       (size_t)T * 8 + 8 + 4 + 8 + 8);
    PQ_CUDA(cudaMemcpyAsync(dD, inst->dist, nn * 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(dF, inst->flow, nn * 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(dDT, DT.data(), nn * 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(dFT, FT.data(), nn * 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(dDd, Dd.data(), n * 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(dFd, Fd.data(), n * 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d.phi, phi.data(), reps * n * 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d.beta, beta.data(), reps * 8, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d.order, order.data(), (size_t)T * cap * 4, cudaMemcpyHostToDevice, q));
    std::vector<int64_t> nob(std::max<size_t>(T, 1), pimqap::kNoBest);
    PQ_CUDA(cudaMemcpyAsync(d.group_best, nob.data(), (size_t)T * 8, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d.single_best, nob.data(), 8, cudaMemcpyHostToDevice, q));
    const int32_t nostop = pimqap::kNoStop;
    const int64_t notarget = std::numeric_limits<int64_t>::max();
    const unsigned long long nons = ~0ull;
    PQ_CUDA(cudaMemcpyAsync(d.stop_epoch, &nostop, 4, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d.target_epoch, &notarget, 8, cudaMemcpyHostToDevice, q));
    PQ_CUDA(cudaMemcpyAsync(d.target_ns, &nons, 8, cudaMemcpyHostToDevice, q));
    PQ_CUDA(pimqap::launch_setup(d, s->bits, q));
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
    for (int k = 0; k < count; ++k) {
        pimqap_status st = pimqap_solve(&insts[k], &params[k], &results[k]);
        if (st != PIMQAP_OK) return st;
    }
    return PIMQAP_OK;
}

}  // extern "C"
