// pimqap_static.cu - pimqap_solve_static: the one-shot solve of pimqap_solve with every device
// buffer (instance copy, replica force matrices and permutations, exchange state) placed in
// one fixed array of device memory that the library reserves when it is loaded, so the call
// itself allocates nothing.
//
// Who needs it: a host program that must not call cudaMalloc while it solves - one that runs
// under a strict device-memory budget owned by another allocator (a framework's caching
// allocator that has claimed the free memory, or a service that admits work by memory it has
// reserved up front), or real-time code that may not take the allocator's locks or its
// latency.  Such a caller gets a solve whose device footprint is fixed when the library loads.
//
// Limits and rules
//   - The array holds kStaticScratchBytes (8 MiB) on every GPU that loads the library, until
//     the process exits.  A solve that needs more (force matrices of all replicas + instance +
//     state) is rejected with PIMQAP_ERR_ARG and a message giving both sizes.
//   - Every call uses the same array and leaves the last call's contents there; each call
//     clears what must start at zero.  Calls that overlap on the same GPU would race on the
//     array: this file serialises the calls of one process per device with a mutex, and a
//     caller that launches work from other processes or libraries into the same context must
//     not overlap them either.
//   - The array's device address is looked up once per device, by the first call on that
//     device, with that device current (cudaGetSymbolAddress on the file-scope symbol; in host
//     code the symbol's name is only a host-side stand-in, never a device address).  Make that
//     first call before any stream capture.
//   - No cudaMalloc, cudaFree, cudaMallocHost, stream, event or graph creation, and no host heap
//     allocation on the success path (small fixed-size host buffers live on the stack).  A
//     failure records its message in the library's last-error slot.
//   - result->device_ms is the host wall time of the launch loop (this entry point creates no
//     CUDA event), so it includes launch and stop-test round trips that pimqap_solve's
//     event-timed figure leaves out.
//   - The force-matrix width is chosen from the cheap per-row bound only (the tighter sorted
//     bound of pimqap_solve needs heap buffers); int64 is used when that bound exceeds int32.
//     Widths do not change results, only memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>

#include "pimqap.h"
#include "pimqap_internal.h"
#include "pimqap_plan.h"

using pimqap::SolveDev;

namespace {

constexpr size_t kStaticScratchBytes = size_t(8) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

void *g_scratch_addr[kMaxDevices] = {};
std::mutex g_device_mutex[kMaxDevices];

pimqap_status fail(pimqap_status st, const char *msg) {
    pimqap::set_last_error(msg);
    return st;
}

using pimqap::detail::carve;
using pimqap::detail::carve_size;

// Small per-call results reduced on the device (no host array of T*R entries is needed).
struct StaticSummary {
    long long best;
    long long arg;
    unsigned long long accepts;
    long long pad;
};

// Pads the raw n x n matrices to rows of ldm (zeros past column n) and writes transposes
// and diagonals, the device layout pimqap_solve builds on the host.
__global__ void static_prepare_kernel(SolveDev d, const int32_t *Draw, const int32_t *Fraw,
                                      int32_t *D_w, int32_t *F_w, int32_t *DT_w, int32_t *FT_w,
                                      int32_t *Dd_w, int32_t *Fd_w) {
    const int n = d.n, ld = d.ldm;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    for (int q = tid; q < n * ld; q += stride) {
        const int i = q / ld, j = q - i * ld;
        const bool in = j < n;
        D_w[q] = in ? Draw[i * n + j] : 0;
        F_w[q] = in ? Fraw[i * n + j] : 0;
        DT_w[q] = in ? Draw[j * n + i] : 0;
        FT_w[q] = in ? Fraw[j * n + i] : 0;
    }
    for (int q = tid; q < n; q += stride) {
        Dd_w[q] = Draw[q * n + q];
        Fd_w[q] = Fraw[q * n + q];
    }
    for (int t = tid; t < d.T; t += stride) d.group_best[t] = pimqap::kNoBest;
    if (tid == 0) {
        *d.single_best = pimqap::kNoBest;
        *d.stop_epoch = pimqap::kNoStop;
        *d.target_epoch = 0x7fffffffffffffffll;
        *d.target_ns = ~0ull;
    }
}

// Replica set-up from one copy per group: every replica of group t starts from the group's
// permutation (CPU_PIM.cpp:143-162), every group has the same beta ladder (:111-119), and rank
// slot l holds replica l (slots past R hold 0, as the reference's zeroed array does).
__global__ void static_replicate_kernel(SolveDev d, const int32_t *group_perms, const double *ladder) {
    const int n = d.n, R = d.R, T = d.T, cap = d.cap;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    const long long reps = (long long)T * R;
    for (long long q = tid; q < reps * n; q += stride) {
        const long long rep = q / n;
        const int i = (int)(q - rep * n);
        d.phi[q] = group_perms[(rep / R) * n + i];
    }
    for (long long q = tid; q < reps; q += stride) d.beta[q] = ladder[q % R];
    for (long long q = tid; q < (long long)T * cap; q += stride) {
        const int l = (int)(q % cap);
        d.order[q] = l < R ? l : 0;
    }
}

__global__ void static_summary_kernel(SolveDev d, StaticSummary *out) {
    __shared__ long long sb[256];
    __shared__ long long sa[256];
    __shared__ unsigned long long sc[256];
    const int reps = d.T * d.R;
    long long best = 0x7fffffffffffffffll, arg = 0;
    unsigned long long acc = 0;
    for (int k = threadIdx.x; k < reps; k += blockDim.x) {
        const long long v = d.bestE[k];
        if (v < best) {
            best = v;
            arg = k;
        }
        acc += d.accepts[k];
    }
    sb[threadIdx.x] = best;
    sa[threadIdx.x] = arg;
    sc[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        // lowest replica index among equal bests, as pimqap_solve picks it
        long long b = sb[0], a = sa[0];
        unsigned long long c = sc[0];
        for (int k = 1; k < (int)blockDim.x; ++k) {
            if (sb[k] < b || (sb[k] == b && sa[k] < a)) {
                b = sb[k];
                a = sa[k];
            }
            c += sc[k];
        }
        out->best = b;
        out->arg = a;
        out->accepts = c;
    }
}

}  // namespace

extern "C" pimqap_status pimqap_solve_static(const pimqap_instance *inst,
                                              const pimqap_params *p, pimqap_result *result) {
    const auto wall0 = std::chrono::steady_clock::now();
    if (!result) return fail(PIMQAP_ERR_ARG, "null result");
    // The checks of pimqap_solve (they build a message only when they fail, so a valid call
    // still allocates nothing), then what this entry point does not run.
    const pimqap_status chk = pimqap::detail::check_params(inst, p);
    if (chk != PIMQAP_OK) return chk;
    if (p->auto_beta) return fail(PIMQAP_ERR_ARG, "automatic beta selection needs pimqap_solve");
    if (p->active_facilities != 0) return fail(PIMQAP_ERR_ARG, "active_facilities needs pimqap_solve");
    if (p->update_rule == PIMQAP_RULE_ONE_SHOT) return fail(PIMQAP_ERR_ARG, "the one-shot rule needs pimqap_solve");
    const int n = inst->n;

    // Instance analysis without heap buffers: symmetry and the per-row force bound.
    const int32_t *F = inst->flow, *D = inst->dist;
    bool sym = true;
    long double A = 0, B = 0, rFmax = 0, cFmax = 0, imax = 0, ebound = 0;
    for (int i = 0; i < n; ++i) {
        long double rf = 0, cf = 0;
        for (int j = 0; j < n; ++j) {
            if (D[i * n + j] != D[j * n + i] || F[i * n + j] != F[j * n + i]) sym = false;
            rf = std::max(rf, std::fabs((long double)F[i * n + j]));
            cf = std::max(cf, std::fabs((long double)F[j * n + i]));
            A = std::max(A, std::fabs((long double)D[i * n + j]));
            B = std::max(B, std::fabs((long double)F[i * n + j]));
        }
        rFmax = std::max(rFmax, rf);
        cFmax = std::max(cFmax, cf);
    }
    for (int i = 0; i < n; ++i) {
        long double rd = 0, cd = 0;
        for (int j = 0; j < n; ++j) {
            rd += std::fabs((long double)D[i * n + j]);
            cd += std::fabs((long double)D[j * n + i]);
        }
        imax = std::max(imax, rd * rFmax + cd * cFmax);
        ebound += rd * rFmax;
    }
    const long double dbound = 4 * imax + 16 * A * B;
    int bits = p->force_bits;
    if (!bits) {
        if (dbound < 2147483647.0L) bits = 32;
        else if (dbound < 4.6e18L && ebound < 4.6e18L) bits = 64;
        else return fail(PIMQAP_ERR_RANGE, "instance values can overflow int64 force matrices");
    }

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PIMQAP_ERR_NO_DEVICE, "no CUDA device");
    const int dev = p->device;
    if (dev < 0 || dev >= ndev || dev >= kMaxDevices) return fail(PIMQAP_ERR_ARG, "bad device ordinal");
    std::lock_guard<std::mutex> lock(g_device_mutex[dev]);
    if (cudaSetDevice(dev) != cudaSuccess) return fail(PIMQAP_ERR_CUDA, "cudaSetDevice failed");
    int major = 0, maxsm = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (major != 10) return fail(PIMQAP_ERR_NO_DEVICE, "the kernels are built for sm_100a only");
    if (pimqap::prepare_kernels() != cudaSuccess) return fail(PIMQAP_ERR_CUDA, "kernel attribute setup failed");
    if (!g_scratch_addr[dev]) {
        void *addr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&addr, g_static_scratch);
        if (e != cudaSuccess || !addr) return fail(PIMQAP_ERR_CUDA, "cudaGetSymbolAddress of the static scratch failed");
        g_scratch_addr[dev] = addr;
    }

    // Launch shape, as pimqap_solve picks it.
    const int T = p->groups, R = p->replicas;
    const int cap = p->rank_slots ? p->rank_slots : std::max(R, 10);
    const int isz = bits / 8, vec = 16 / isz;
    const int npad = (n + 3) & ~3;
    int lds = npad;
    if ((lds / vec) % 2 == 0) lds += vec;
    const int threads = p->threads_per_block ? p->threads_per_block : (n <= 64 ? 64 : (n <= 128 ? 128 : 256));
    auto rows_per_cta = [&](int c) { return (((n + c - 1) / c) + 3) & ~3; };
    int cl = 0;
    for (int c : {1, 2, 4}) {
        if (p->cluster_size && c != p->cluster_size) continue;
        if (pimqap::epoch_smem_bytes(n, rows_per_cta(c), lds, c, bits) <= (size_t)maxsm) {
            cl = c;
            break;
        }
    }
    if (!cl) return fail(PIMQAP_ERR_ARG, "force matrix does not fit a 4-CTA cluster");
    const int rpc = rows_per_cta(cl);
    const int ldm = std::max(npad, cl * rpc);
    const size_t smem = pimqap::epoch_smem_bytes(n, rpc, lds, cl, bits);

    const size_t reps = (size_t)T * R, nn = (size_t)n * ldm, nraw = (size_t)n * n;
    const size_t need = carve_size(reps * (size_t)n * npad * isz) + 4 * carve_size(nn * 4) +
                        2 * carve_size(nraw * 4) +
                        2 * carve_size((size_t)n * 4) + 2 * carve_size(reps * n * 4) +
                        4 * carve_size(reps * 8) + carve_size((size_t)T * cap * 4) +
                        4 * carve_size((size_t)T * 8) + 8 * carve_size(8) + carve_size(sizeof(StaticSummary)) +
                        carve_size((size_t)T * n * 4) + carve_size((size_t)R * 8);
    if (need > kStaticScratchBytes) {
        char msg[160];
        std::snprintf(msg, sizeof msg,
                      "solve needs %zu bytes of device memory; the static scratch holds %zu (8 MiB)",
                      need, kStaticScratchBytes);
        return fail(PIMQAP_ERR_ARG, msg);
    }

    char *base = reinterpret_cast<char *>(g_scratch_addr[dev]);
    char *cur = base;
    SolveDev d{};
    d.n = n; d.R = R; d.T = T; d.cap = cap; d.spe = p->sweeps_per_exchange;
    d.ldg = npad; d.lds = lds; d.ldm = ldm; d.rpc = rpc;
    d.goal = p->goal;
    d.seed = p->seed;
    d.I = carve<char>(cur, reps * (size_t)n * npad * isz);
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
    StaticSummary *dsum = carve<StaticSummary>(cur, 1);
    int32_t *rawD = carve<int32_t>(cur, nraw), *rawF = carve<int32_t>(cur, nraw);
    int32_t *group_perms = carve<int32_t>(cur, (size_t)T * n);
    double *dladder = carve<double>(cur, R);

    const cudaStream_t q = 0;   // the legacy default stream: nothing is created per call
#define PQS_CUDA(x)                                                     \
    do {                                                                \
        if ((x) != cudaSuccess) return fail(PIMQAP_ERR_CUDA, #x " failed"); \
    } while (0)
    PQS_CUDA(cudaMemsetAsync(base, 0, need, q));   // the previous call's contents are cleared
    PQS_CUDA(cudaMemcpy(rawD, D, nraw * 4, cudaMemcpyHostToDevice));
    PQS_CUDA(cudaMemcpy(rawF, F, nraw * 4, cudaMemcpyHostToDevice));
    static_prepare_kernel<<<64, 256, 0, q>>>(d, rawD, rawF, dD, dF, dDT, dFT, dDd, dFd);
    PQS_CUDA(cudaGetLastError());

    // Host set-up with fixed-size stack buffers: each group's shuffle (drawn group after group
    // from one stream), uploaded a chunk of groups per copy, and the beta ladder once; a kernel
    // gives every replica its group's permutation and ladder slot.
    const double beta0 = p->beta_internal ? p->beta_max : p->beta_max * 1.44269504089;
    pimqap::detail::ShuffleEngine eng;
    eng.seed = p->seed;
    constexpr int kStageInts = 4096;                  // 16 KB of permutations per copy
    int32_t stage[kStageInts];
    const int per_copy = kStageInts / n;             // >= 16 groups, since n <= 256
    for (int t0 = 0; t0 < T; t0 += per_copy) {
        const int cnt = std::min(per_copy, T - t0);
        for (int k = 0; k < cnt; ++k) pimqap::detail::shuffle_group(eng, n, stage + (size_t)k * n);
        PQS_CUDA(cudaMemcpy(group_perms + (size_t)t0 * n, stage, (size_t)cnt * n * 4, cudaMemcpyHostToDevice));
    }
    double ladder[PIMQAP_MAX_REPLICAS];
    double running = beta0;
    for (int l = R - 1; l >= 0; --l) {
        ladder[l] = running;
        running /= p->beta_ratio;
    }
    PQS_CUDA(cudaMemcpy(dladder, ladder, (size_t)R * 8, cudaMemcpyHostToDevice));
    static_replicate_kernel<<<64, 256, 0, q>>>(d, group_perms, dladder);
    PQS_CUDA(cudaGetLastError());
    PQS_CUDA(pimqap::launch_setup(d, bits, q));
    PQS_CUDA(cudaStreamSynchronize(q));

    // Mega-iterations, one epoch launch each; goal and timeout are checked every few launches,
    // the timeout counted from here as pimqap_solve counts it from the start of its run loop.
    const auto run0 = std::chrono::steady_clock::now();
    const int check_every = p->megaiters_per_launch > 0 ? p->megaiters_per_launch : 50;
    int64_t left = p->max_megaiters;
    bool stopped_goal = false;
    while (left > 0) {
        const int g = (int)std::min<int64_t>(left, check_every);
        for (int k = 0; k < g; ++k) PQS_CUDA(pimqap::launch_epoch(d, bits, cl, sym, false, threads, smem, q));
        int32_t stop = 0;
        PQS_CUDA(cudaMemcpy(&stop, d.stop_epoch, 4, cudaMemcpyDeviceToHost));
        left -= g;
        if (stop != pimqap::kNoStop) {
            stopped_goal = true;
            break;
        }
        if (p->timeout_s > 0 &&
            std::chrono::duration<double>(std::chrono::steady_clock::now() - run0).count() >= p->timeout_s)
            break;
    }
    static_summary_kernel<<<1, 256, 0, q>>>(d, dsum);
    PQS_CUDA(cudaGetLastError());
    StaticSummary sum{};
    int32_t epoch0 = 0, err = 0;
    int64_t single = 0, tepoch = 0;
    unsigned long long tns = 0, sns = 0;
    PQS_CUDA(cudaMemcpy(&sum, dsum, sizeof sum, cudaMemcpyDeviceToHost));
    PQS_CUDA(cudaMemcpy(&epoch0, d.epoch, 4, cudaMemcpyDeviceToHost));
    PQS_CUDA(cudaMemcpy(&err, d.error, 4, cudaMemcpyDeviceToHost));
    PQS_CUDA(cudaMemcpy(&single, d.single_best, 8, cudaMemcpyDeviceToHost));
    PQS_CUDA(cudaMemcpy(&tepoch, d.target_epoch, 8, cudaMemcpyDeviceToHost));
    PQS_CUDA(cudaMemcpy(&tns, d.target_ns, 8, cudaMemcpyDeviceToHost));
    PQS_CUDA(cudaMemcpy(&sns, d.start_ns, 8, cudaMemcpyDeviceToHost));
    if (err) return fail(PIMQAP_ERR_DEVICE, "device check failed");
    int32_t *perm_dst = result->best_perm;
    int64_t *energy_dst = result->final_energies;
    std::memset(result, 0, sizeof(*result));
    result->best_perm = perm_dst;
    result->final_energies = energy_dst;
    if (perm_dst)
        PQS_CUDA(cudaMemcpy(perm_dst, d.best_phi + (size_t)sum.arg * n, (size_t)n * 4, cudaMemcpyDeviceToHost));
    if (energy_dst) PQS_CUDA(cudaMemcpy(energy_dst, d.E, reps * 8, cudaMemcpyDeviceToHost));
    result->beta_max_used = beta0;
    result->beta_ratio_used = p->beta_ratio;
#undef PQS_CUDA
    const auto wall1 = std::chrono::steady_clock::now();
    result->best_energy = std::min<int64_t>(sum.best, single);
    result->target_megaiter = (tepoch == 0x7fffffffffffffffll) ? -1 : tepoch;
    result->time_to_target_ms = (result->target_megaiter >= 0 && tns != ~0ull && tns >= sns) ? (double)(tns - sns) * 1e-6 : -1.0;
    result->megaiters_done = epoch0;
    result->updates = (int64_t)epoch0 * p->sweeps_per_exchange * n * (int64_t)reps;
    result->sweeps = result->updates / n;
    result->proposals = result->sweeps * ((int64_t)n * (n - 1) / 2);
    result->accepts = (int64_t)sum.accepts;
    // host wall time of the launch loop: this entry point creates no CUDA events
    result->device_ms = std::chrono::duration<double, std::milli>(wall1 - run0).count();
    result->wall_ms = std::chrono::duration<double, std::milli>(wall1 - wall0).count();
    result->force_bits = bits;
    result->cluster_size = cl;
    // pimqap_solve's rule: a timeout is the stop only when mega-iterations were left to run
    result->stopped_by = stopped_goal ? 1 : ((p->timeout_s > 0 && epoch0 < p->max_megaiters) ? 2 : 0);
    result->h2d_bytes = (int64_t)(2 * nraw * 4 + (size_t)T * n * 4 + (size_t)R * 8);
    result->d2h_bytes = (int64_t)(sizeof sum + 4 + 4 + 8 + 8 + 8 + 8 + (perm_dst ? (size_t)n * 4 : 0));
    return PIMQAP_OK;
}
