// pimqap_kernels.cu - sm_100a kernels of the parallel-tempering p-dit QAP solver.
//
// Kernels
//   init_force_kernel   I[i][a] = -sum_j (D[i][j] F[a][phi(j)] + D[j][i] F[phi(j)][a])
//                       (reference setup(), CPU-PIM/CPU_PIM.cpp:164-181), tiled integer GEMM
//   init_energy_kernel  E = -1/2 sum_i I[i][phi(i)]  (equals CPU_PIM.cpp:184-192 exactly)
//   init_exchange_kernel  tracking/exchange of mega-iteration 0 (CPU_PIM.cpp:293-344)
//   epoch_kernel        spe sweeps of one replica (doMegaItera, CPU_PIM.cpp:195-290) with the
//                       replica's force matrix resident in shared memory, split by rows over a
//                       thread-block cluster when it does not fit one CTA; then the last
//                       replica of each group to finish runs the group's tracking + exchange.
//
// One p-dit update of location i (a = phi(i)) in the epoch kernel:
//   1. every CTA computes the swap deltas of the candidate locations j it owns (row j of I
//      is local; row i is read from the owning CTA through distributed shared memory) and
//      scatters dE[b], b = phi(j), plus its warp maxima, into every CTA of the cluster;
//   2. cluster barrier;
//   3. every CTA redundantly (bit-identical inputs and code) forms the heat-bath weights
//      exp2(beta dE) above the reference's cutoff, a double-precision prefix sum in b order,
//      and picks the first b whose prefix reaches r * total;
//   4. on a swap, every CTA applies the rank-2 force update to the rows it owns, then a
//      cluster barrier publishes the new rows.
// Rejected updates cost one barrier; double-buffered delta / maxima slots make that safe.
#include <cooperative_groups.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "pimqap_internal.h"
#include "pimqap_weights.cuh"

namespace cg = cooperative_groups;

namespace pimqap {

// ------------------------------------------------------------------ helpers

template <class IT> struct Unsigned;
template <> struct Unsigned<int32_t> { using type = uint32_t; };
template <> struct Unsigned<int64_t> { using type = uint64_t; };

template <class IT> struct alignas(16) Vec {
    static constexpr int kN = 16 / sizeof(IT);
    IT v[kN];
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// Shared memory the tracking / exchange step stages a group in (track_exchange): energies,
// bests and betas of up to kMaxReplicas replicas and their rank slots (+ slot cap-1).
constexpr int kMaxReplicas = 64;
constexpr size_t kExchangeScratchBytes = (size_t)kMaxReplicas * (8 + 8 + 8) + (kMaxReplicas + 1) * 4;

// Offsets (bytes) of the epoch kernel's shared-memory sections.
//   I       rpc rows of the replica's force matrix (row stride lds)
//   phi, inv, bphi, Dd, Fd    permutation, inverse, best permutation, diagonals of D and F
//   A, B    [2][npad] receive buffers of the two delta halves (double-buffered by update)
//   Drow, DTrow  [2][rpc]  D[i][own rows], D[own rows][i] for the current / next location i
//   Frow, FTrow  [2][npad] F[a][*], F[*][a] for a = phi(i), current / next
//   Dj, DTj, Fb, FTb        the same rows for the partner j / facility b of an accepted swap
//   red, wsum, r, misc, bar  reductions, the random numbers of a sweep, pick, mbarriers
struct SmemLayout {
    size_t I, phi, inv, bphi, Dd, Fd, A, B, Drow, DTrow, Frow, FTrow, Dj, DTj, Fb, FTb;
    size_t u1, u2, red, wsum, r, misc, bar, total;
    __host__ __device__ SmemLayout(int n, int rpc, int lds, int cluster, int isz) {
        const size_t npad = (size_t)((n + 3) & ~3);
        const size_t rp = (size_t)rpc;
        size_t o = 0;
        I = o;     o = align16(o + rp * lds * isz);
        phi = o;   o = align16(o + npad * 4);
        inv = o;   o = align16(o + npad * 4);
        bphi = o;  o = align16(o + npad * 4);
        Dd = o;    o = align16(o + npad * 4);
        Fd = o;    o = align16(o + npad * 4);
        A = o;     o = align16(o + 2 * npad * isz);
        B = o;     o = align16(o + (cluster > 1 ? 2 * npad * isz : 0));
        Drow = o;  o = align16(o + 2 * rp * 4);
        DTrow = o; o = align16(o + 2 * rp * 4);
        Frow = o;  o = align16(o + 2 * npad * 4);
        FTrow = o; o = align16(o + 2 * npad * 4);
        Dj = o;    o = align16(o + rp * 4);
        DTj = o;   o = align16(o + rp * 4);
        Fb = o;    o = align16(o + npad * 4);
        FTb = o;   o = align16(o + npad * 4);
        u1 = o;    o = align16(o + rp * isz);
        u2 = o;    o = align16(o + rp * isz);
        red = o;   o = align16(o + kMaxWarps * 8);
        wsum = o;  o = align16(o + kMaxWarps * sizeof(double));
        r = o;     o = align16(o + npad * sizeof(double));   // r of each update of a sweep
        misc = o;  o = align16(o + 4 * sizeof(int));
        bar = o;   o = align16(o + 2 * sizeof(unsigned long long));
        total = o;
    }
};

size_t epoch_smem_bytes(int n, int rpc, int lds, int cluster, int bits) {
    return SmemLayout(n, rpc, lds, cluster, bits / 8).total;
}

size_t exchange_scratch_bytes() { return 16 + kExchangeScratchBytes; }

// Philox4x32-10 (Salmon et al., SC'11): words 0 and 1 of the block for counter c, key k.
__device__ __forceinline__ void philox_2words(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                              uint32_t k0, uint32_t k1, uint32_t &w0,
                                              uint32_t &w1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    w0 = c0;
    w1 = c1;
}

// All four words of the block (the lumped draw of a clique-flow update).
__device__ __forceinline__ void philox_4words(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                              uint32_t k0, uint32_t k1, uint32_t w[4]) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    w[0] = c0; w[1] = c1; w[2] = c2; w[3] = c3;
}

// Facility of a lumped clique-flow move (CPU_PIM_tai256c.cpp:326): act + uniform_int(range)
// by Lemire's method on words 2 and 3 of the update's block, then on blocks whose counter
// word 3 is group + 0x10000 m, m = 1, 2, ... (one thread).
__device__ __noinline__ int lumped_facility(uint32_t loc, uint32_t sweep, uint32_t rep, uint32_t grp,
                                            uint32_t k0, uint32_t k1, int act, uint32_t range) {
    uint32_t w[4];
    philox_4words(loc, sweep, rep, grp, k0, k1, w);
    uint32_t k = 0;
    auto word = [&]() -> uint32_t {
        uint32_t v;
        if (k < 2) {
            v = w[2 + k];
        } else {
            const uint32_t m = (k - 2) / 4 + 1;
            if ((k - 2) % 4 == 0) philox_4words(loc, sweep, rep, grp + 0x10000u * m, k0, k1, w);
            v = w[(k - 2) % 4];
        }
        ++k;
        return v;
    };
    unsigned long long product = (unsigned long long)word() * range;
    uint32_t low = (uint32_t)product;
    if (low < range) {
        const uint32_t threshold = (0u - range) % range;
        while (low < threshold) {
            product = (unsigned long long)word() * range;
            low = (uint32_t)product;
        }
    }
    return act + (int)(product >> 32);
}

// std::generate_canonical<double, 53> over two 32-bit words (CPU_PIM.cpp:212):
// (w0 + w1 * 2^32) rounded once to double, times 2^-64, clamped below 1.
__device__ __forceinline__ double canonical53(uint32_t w0, uint32_t w1) {
    const double s = __dadd_rn((double)w0, __dmul_rn((double)w1, 4294967296.0));
    double r = __dmul_rn(s, 0x1p-64);
    if (r >= 1.0) r = 0x1.fffffffffffffp-1;
    return r;
}

// (int)x of CPU_PIM.cpp:235: truncation toward zero, the most negative value outside range.
__device__ __forceinline__ long long cutoff_trunc(double x) {
    if (!(x > -9223372036854775808.0) || !(x < 9223372036854775808.0))
        return (long long)0x8000000000000000ull;
    return __double2ll_rz(x);
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <int CL> __device__ __forceinline__ void cluster_barrier() {
    if constexpr (CL == 1) {
        __syncthreads();
    } else {
        asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
                     "barrier.cluster.wait.acquire.aligned;" ::: "memory");
    }
}

template <class IT> __device__ __forceinline__ IT warp_max(IT v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        IT w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}
// 32-bit values: one warp-wide reduction instruction (redux.sync) instead of five shuffles.
template <> __device__ __forceinline__ int32_t warp_max<int32_t>(int32_t v) {
    return __reduce_max_sync(0xffffffffu, v);
}

// The largest of the nwarps (<= 32) warp maxima in s_red, all >= 0, in every thread of a warp:
// 32-bit values by one load per lane and a warp reduction, wider ones by a loop.
template <class IT> __device__ __forceinline__ IT block_max(const IT *s_red, int nwarps, int lane) {
    if constexpr (sizeof(IT) == 4) {
        return __reduce_max_sync(0xffffffffu, lane < nwarps ? s_red[lane] : (IT)0);
    } else {
        IT M = s_red[0];
        for (int w = 1; w < nwarps; ++w) M = s_red[w] > M ? s_red[w] : M;
        return M;
    }
}

// Sum of eight doubles as a pairwise tree (three dependent adds).
__device__ __forceinline__ double tree8(const double (&v)[8]) {
    return __dadd_rn(__dadd_rn(__dadd_rn(v[0], v[1]), __dadd_rn(v[2], v[3])),
                     __dadd_rn(__dadd_rn(v[4], v[5]), __dadd_rn(v[6], v[7])));
}

// The weight total of an update from the nwarps (<= 8) per-warp totals in s_wsum, and the
// part of it before warp `warp`: independent loads summed as pairwise trees instead of a chain
// of dependent adds (adding the zeros past nwarps is exact).  The weights are double sums in
// an order of this kernel's choosing either way; the reference sums them in sequence in long
// double (CPU_PIM.cpp:240-245), so a decision can differ from it only where r * total falls
// within a few ulp of a prefix boundary, whatever the order.
__device__ __forceinline__ void weight_totals(const double *s_wsum, int nwarps, int warp, double &base,
                                              double &total) {
    double v[8], b[8];
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        v[w] = w < nwarps ? s_wsum[w] : 0.0;
        b[w] = w < warp ? v[w] : 0.0;
    }
    total = tree8(v);
    base = tree8(b);
}

// ---- shared::cluster addressing, mbarriers, asynchronous remote stores, async copies

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint32_t cluster_addr(uint32_t cta_addr, int rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(cta_addr), "r"(rank));
    return r;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
// Ends an mbarrier's life, so the same shared-memory word can be initialised again for the
// next replica a persistent worker runs.
__device__ __forceinline__ void mbar_inval(uint32_t bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up (returns false) after limit_ns of global time.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity,
                                                  unsigned long long limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
    return true;
}
__device__ __forceinline__ void st_async(uint32_t dst, int32_t v, uint32_t bar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b32 [%0], %1, [%2];"
                 ::"r"(dst), "r"(v), "r"(bar) : "memory");
}
__device__ __forceinline__ void st_async(uint32_t dst, int64_t v, uint32_t bar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b64 [%0], %1, [%2];"
                 ::"r"(dst), "l"(v), "r"(bar) : "memory");
}
__device__ __forceinline__ void st_async16(uint32_t dst, const Vec<int32_t> &v, uint32_t bar) {
    asm volatile(
        "st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];"
        ::"r"(dst), "r"(v.v[0]), "r"(v.v[1]), "r"(v.v[2]), "r"(v.v[3]), "r"(bar) : "memory");
}
__device__ __forceinline__ void st_async16(uint32_t dst, const Vec<int64_t> &v, uint32_t bar) {
    asm volatile(
        "st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.b64 [%0], {%1, %2}, [%3];"
        ::"r"(dst), "l"(v.v[0]), "l"(v.v[1]), "r"(bar) : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem)), "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Copies rows of 16-byte chunks global -> shared with cp.async, spread over the CTA.
//   D slice:  nD chunks from gD to sD (and gDT to sDT when two)
//   F row:    nF chunks from gF to sF (and gFT to sFT)
template <bool SYM>
__device__ __forceinline__ void prefetch_rows(int tid, int BT, int nD, const int32_t *gD,
                                              const int32_t *gDT, int32_t *sD, int32_t *sDT,
                                              int nF, const int32_t *gF, const int32_t *gFT,
                                              int32_t *sF, int32_t *sFT) {
    const int per = SYM ? (nD + nF) : 2 * (nD + nF);
    for (int q = tid; q < per; q += BT) {
        int k = q;
        if (k < nD) { cp_async16(sD + 4 * k, gD + 4 * k); continue; }
        k -= nD;
        if (k < nF) { cp_async16(sF + 4 * k, gF + 4 * k); continue; }
        k -= nF;
        if constexpr (!SYM) {
            if (k < nD) { cp_async16(sDT + 4 * k, gDT + 4 * k); continue; }
            k -= nD;
            cp_async16(sFT + 4 * k, gFT + 4 * k);
        }
    }
    cp_async_commit();
}

// ------------------------------------------------------------------ tracking + exchange

// Best tracking, replica exchange and goal test of group g at the start of mega-iteration
// e_next (CPU_PIM.cpp:295-348).  Runs on one thread after every replica of the group has
// finished its sweeps.  With `scratch` (kExchangeScratchBytes of shared memory that nothing
// else uses meanwhile) the group's energies, bests, betas and rank order are first read
// through L2 with independent loads and the bubble pass runs on those copies, so its chain of
// rank-slot reads and writes stays in shared memory; without it, it works on global memory.
__device__ void track_exchange(const SolveDev &s, int g, int e_next, unsigned char *scratch = nullptr) {
    const int R = s.R, cap = s.cap;
    int64_t *gE = s.E + (size_t)g * R;
    int64_t *gbestE = s.bestE + (size_t)g * R;
    double *gbeta = s.beta + (size_t)g * R;
    int32_t *gorder = s.order + (size_t)g * cap;
    const bool staged = scratch != nullptr && R <= kMaxReplicas;
    volatile int64_t *E, *bestE;
    volatile double *beta;
    volatile int32_t *order;
    int hi;                                                  // index of rank slot cap-1
    if (staged) {
        int64_t *sE = reinterpret_cast<int64_t *>(scratch);
        int64_t *sB = sE + kMaxReplicas;
        double *sb = reinterpret_cast<double *>(sB + kMaxReplicas);
        int32_t *so = reinterpret_cast<int32_t *>(sb + kMaxReplicas);
#pragma unroll 8
        for (int l = 0; l < R; ++l) {
            sE[l] = __ldcg((const long long *)gE + l);
            sB[l] = __ldcg((const long long *)gbestE + l);
            sb[l] = __ldcg(gbeta + l);
            so[l] = __ldcg(gorder + l);
        }
        hi = cap - 1 < R ? cap - 1 : R;                      // slots R .. cap-2 are never read
        if (hi == R) so[R] = __ldcg(gorder + cap - 1);
        E = sE; bestE = sB; beta = sb; order = so;
    } else {
        E = gE; bestE = gbestE; beta = gbeta; order = gorder;
        hi = cap - 1;
    }
    int tss = *((volatile int32_t *)s.tss + g) + 1;          // :295
    int64_t gb = *((volatile int64_t *)s.group_best + g);
    bool found = false;
    for (int l = 0; l < R; ++l) {                            // :297-314
        const int64_t b = bestE[l];
        if (b < gb) {
            found = true;
            gb = b;
            tss = 0;
            if (s.ev.log) {
                const unsigned idx = atomicAdd(s.ev.count, 1u);
                if (idx < s.ev.cap) s.ev.log[idx] = EventDev{e_next, g, l, -1, b, globaltimer_ns(), s.ev.tag, 0};
            }
        }
    }
    if (found) atomicMin((long long *)s.single_best, (long long)gb);
    bool ok = true;
    for (int l = 0; l < R - 1; ++l) {                        // :324-337
        const int i1 = order[l], i2 = order[l + 1];
        if ((unsigned)i1 >= (unsigned)R || (unsigned)i2 >= (unsigned)R) {   // never in a valid state
            ok = false;
            break;
        }
        const double e1 = (double)E[i1], e2 = (double)E[i2];
        if (e1 < e2) {
            order[l] = i2;
            order[l + 1] = i1;
            const double tb = beta[i1];
            beta[i1] = beta[i2];
            beta[i2] = tb;
            if (i2 == R - 1) tss = 0;                        // replica index, as :333
        }
    }
    if (ok && tss > 100) {                                   // :339-344, slot cap-1
        const int i1 = order[hi], i2 = order[0];
        if ((unsigned)i1 >= (unsigned)R || (unsigned)i2 >= (unsigned)R) {
            ok = false;
        } else {
            order[hi] = i2;
            order[0] = i1;
            const double tb = beta[i1];
            beta[i1] = beta[i2];
            beta[i2] = tb;
        }
    }
    if (staged) {   // the copies back (also after a failed check: nothing else has changed)
        for (int l = 0; l < R; ++l) {
            gbeta[l] = beta[l];
            gorder[l] = order[l];
        }
        if (hi == R) gorder[cap - 1] = order[R];
    }
    if (!ok) {
        atomicOr(s.error, kErrShape);
        return;
    }
    s.tss[g] = tss;
    s.group_best[g] = gb;
    __threadfence();
    const long long sb = atomicAdd((unsigned long long *)s.single_best, 0ull);
    if (sb <= s.goal) {                                      // :346
        atomicMin(s.stop_epoch, e_next);
        atomicMin((long long *)s.target_epoch, (long long)e_next);
        atomicMin(s.target_ns, globaltimer_ns());
    }
}

// ------------------------------------------------------------------ setup kernels

template <class IT>
__global__ void __launch_bounds__(256) init_force_kernel(SolveDev s) {
    __shared__ int32_t sD[16][17], sDT[16][17], sFp[16][17], sFTp[16][17];
    const int n = s.n;
    const int rep = blockIdx.x;                // grid: (replicas, column tiles, row tiles)
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = blockIdx.z * 16 + ty;        // location (row of I)
    const int a = blockIdx.y * 16 + tx;        // facility (column of I)
    const int arow = blockIdx.y * 16 + ty;     // facility row staged by this thread
    const int32_t *phi = s.phi + (size_t)rep * n;
    long long acc = 0;
    for (int j0 = 0; j0 < n; j0 += 16) {
        const int j = j0 + tx;
        const bool jok = j < n;
        const int pj = jok ? phi[j] : 0;
        const int ld = s.ldm;
        sD[ty][tx] = (i < n && jok) ? s.D[i * ld + j] : 0;
        sDT[ty][tx] = (i < n && jok) ? s.DT[i * ld + j] : 0;
        sFp[ty][tx] = (arow < n && jok) ? s.F[arow * ld + pj] : 0;
        sFTp[ty][tx] = (arow < n && jok) ? s.FT[arow * ld + pj] : 0;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k)
            acc += (long long)sD[ty][k] * sFp[tx][k] + (long long)sDT[ty][k] * sFTp[tx][k];
        __syncthreads();
    }
    IT *I = reinterpret_cast<IT *>(s.I) + (size_t)rep * n * s.ldg;
    if (i < n && a < s.ldg) I[(size_t)i * s.ldg + a] = (a < n) ? (IT)(-acc) : (IT)0;
}

template <class IT>
__global__ void __launch_bounds__(256) init_energy_kernel(SolveDev s) {
    __shared__ long long part[kMaxWarps];
    const int n = s.n;
    const int rep = blockIdx.x;
    const IT *I = reinterpret_cast<const IT *>(s.I) + (size_t)rep * n * s.ldg;
    const int32_t *phi = s.phi + (size_t)rep * n;
    long long acc = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        acc += (long long)I[(size_t)i * s.ldg + phi[i]];
        s.best_phi[(size_t)rep * n + i] = phi[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
        s.E[rep] = -t / 2;                 // sum_i I[i][phi(i)] = -2E exactly
        s.bestE[rep] = kNoBest;
        s.accepts[rep] = 0ull;
    }
}

__global__ void init_exchange_kernel(SolveDev s) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g == 0) *s.start_ns = globaltimer_ns();
    if (g < s.T) track_exchange(s, g, 0);
}

// ------------------------------------------------------------------ the epoch kernel

// Limit of one bounded wait for a peer CTA's delta halves.  A healthy wait lasts
// microseconds; after a timeout the CTA records kErrTimeout and stops sweeping.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;

// A replica worker: the whole CTA (bar == 0, __syncthreads) or a group of warps of it that
// synchronises on its own named barrier (bar = 1..15), so several workers share one CTA.
struct Grp {
    int tid, BT, lane, warp, nwarps, bar;
    __device__ __forceinline__ void sync() const {
        if (bar == 0) __syncthreads();
        else asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(BT) : "memory");
    }
    __device__ __forceinline__ bool sync_or(bool v) const {
        if (bar == 0) return __syncthreads_or(v) != 0;
        uint32_t r;
        asm volatile(
            "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\t"
            "bar.red.or.pred q, %2, %3, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
            : "=r"(r)
            : "r"((uint32_t)v), "r"(bar), "r"(BT)
            : "memory");
        return r != 0;
    }
};

template <int CL> __device__ __forceinline__ void cluster_sync(const Grp &G) {
    if constexpr (CL == 1) G.sync();
    else cluster_barrier<CL>();
}

// A replica's best fell below goal_print during a sweep of mega-iteration e (the reference
// prints the replica and its permutation, CPU_PIM.cpp:271-282).  One thread claims a
// permutation slot and appends the event; the CTA fills the slot after its next barrier.
// Returns the slot, or -1 when the permutation store is full.
__device__ __forceinline__ int goal_print_claim(const EventLink &v, int g, int l, int e, int64_t E) {
    if (!v.log) return -1;
    const unsigned slot = atomicAdd(v.count + 1, 1u);
    const bool stored = slot < v.pcap;
    const unsigned idx = atomicAdd(v.count, 1u);
    if (idx < v.cap)
        v.log[idx] = EventDev{e, g, l, stored ? (int32_t)slot : -2, E, globaltimer_ns(), v.tag, 0};
    return stored ? (int)slot : -1;
}

// One epoch of replica rep: load its state into shared memory, spe sweeps (doMegaItera,
// CPU_PIM.cpp:195-290), store the state back.  With CL > 1 this CTA is rank `rank` of the
// replica's cluster and G is the whole CTA.  Replica state is read through L2 (__ldcg): the
// previous epoch may have run on another SM.  Returns false when a bounded wait gave up.
template <class IT, int CL, bool SYM, bool GP = false>
__device__ bool replica_epoch(const SolveDev &s, int rep, int rank, int e, const Grp &G,
                              unsigned char *smem) {
    using U = typename Unsigned<IT>::type;
    constexpr int VEC = Vec<IT>::kN;
    const int n = s.n;
    const int tid = G.tid, BT = G.BT, lane = G.lane, warp = G.warp, nwarps = G.nwarps;
    const int g = rep / s.R, l = rep - g * s.R;

    const int rpc = s.rpc, lds = s.lds, ldm = s.ldm;
    const int row0 = rank * rpc;
    const int rows = max(0, min(rpc, n - row0));
    const int npad = (n + 3) & ~3;
    const SmemLayout L(n, rpc, lds, CL, (int)sizeof(IT));
    IT *sI = reinterpret_cast<IT *>(smem + L.I);
    int32_t *s_phi = reinterpret_cast<int32_t *>(smem + L.phi);
    int32_t *s_inv = reinterpret_cast<int32_t *>(smem + L.inv);
    int32_t *s_bphi = reinterpret_cast<int32_t *>(smem + L.bphi);
    int32_t *s_Dd = reinterpret_cast<int32_t *>(smem + L.Dd);
    int32_t *s_Fd = reinterpret_cast<int32_t *>(smem + L.Fd);
    IT *s_A = reinterpret_cast<IT *>(smem + L.A);
    IT *s_B = reinterpret_cast<IT *>(smem + L.B);
    int32_t *s_Drow = reinterpret_cast<int32_t *>(smem + L.Drow);
    int32_t *s_DTrow = reinterpret_cast<int32_t *>(smem + L.DTrow);
    int32_t *s_Frow = reinterpret_cast<int32_t *>(smem + L.Frow);
    int32_t *s_FTrow = reinterpret_cast<int32_t *>(smem + L.FTrow);
    int32_t *s_Dj = reinterpret_cast<int32_t *>(smem + L.Dj);
    int32_t *s_DTj = reinterpret_cast<int32_t *>(smem + L.DTj);
    int32_t *s_Fb = reinterpret_cast<int32_t *>(smem + L.Fb);
    int32_t *s_FTb = reinterpret_cast<int32_t *>(smem + L.FTb);
    IT *s_u1 = reinterpret_cast<IT *>(smem + L.u1);          // row factors of the accepted swap
    IT *s_u2 = reinterpret_cast<IT *>(smem + L.u2);
    IT *s_red = reinterpret_cast<IT *>(smem + L.red);
    double *s_wsum = reinterpret_cast<double *>(smem + L.wsum);
    double *s_r = reinterpret_cast<double *>(smem + L.r);
    int *s_misc = reinterpret_cast<int *>(smem + L.misc);   // [0] pick, [1] improved-at, [2] error, [3] goal-print slot
    unsigned long long *s_bar = reinterpret_cast<unsigned long long *>(smem + L.bar);
    const int nDc = rpc / 4, nFc = npad / 4;                 // 16-byte chunks of a D slice / F row

    // ---- load the replica and prefetch the rows of update 0
    {
        const IT *gI = reinterpret_cast<const IT *>(s.I) + ((size_t)rep * n + row0) * s.ldg;
        const int nvg = s.ldg / VEC;
        for (int idx = tid; idx < rows * nvg; idx += BT) {
            const int k = idx / nvg, v = idx - k * nvg;
            const int4 w = __ldcg(reinterpret_cast<const int4 *>(gI + (size_t)k * s.ldg + v * VEC));
            *reinterpret_cast<int4 *>(sI + (size_t)k * lds + v * VEC) = w;
        }
        const int32_t *gphi = s.phi + (size_t)rep * n;
        for (int q = tid; q < npad; q += BT) {
            // an entry outside [0, n) would index out of range: clamp it and flag the error
            int p = q < n ? __ldcg(gphi + q) : 0;
            if ((unsigned)p >= (unsigned)n) {
                atomicOr(s.error, kErrBadPerm);
                p = 0;
            }
            s_phi[q] = p;
            s_bphi[q] = p;
            s_inv[q] = 0;
            s_Dd[q] = q < n ? __ldcg(s.Ddiag + q) : 0;
            s_Fd[q] = q < n ? __ldcg(s.Fdiag + q) : 0;
        }
        if (tid == 0) {
            s_misc[0] = 0x7fffffff;
            s_misc[1] = -1;
            s_misc[2] = 0;
            if constexpr (CL > 1) {
                mbar_init(smem_u32(&s_bar[0]), 1);
                mbar_init(smem_u32(&s_bar[1]), 1);
                mbar_fence_init();
            }
        }
        G.sync();
        const int a0 = s_phi[0];
        prefetch_rows<SYM>(tid, BT, nDc, s.D + row0, s.DT + row0, s_Drow, s_DTrow, nFc,
                           s.F + (size_t)a0 * ldm, s.FT + (size_t)a0 * ldm, s_Frow, s_FTrow);
    }
    for (int q = tid; q < n; q += BT) s_inv[s_phi[q]] = q;
    cp_async_wait_all();
    cluster_sync<CL>(G);   // every CTA of the cluster is resident, initialised, rows loaded

    // shared::cluster addresses of every CTA's receive buffers and mbarriers
    uint32_t A_at[CL], B_at[CL], bar_at[CL];
    if constexpr (CL > 1) {
#pragma unroll
        for (int r = 0; r < CL; ++r) {
            A_at[r] = cluster_addr(smem_u32(s_A), r);
            B_at[r] = cluster_addr(smem_u32(s_B), r);
            bar_at[r] = cluster_addr(smem_u32(s_bar), r);
        }
    }
    const uint32_t tx_bytes = (uint32_t)((npad + n) * sizeof(IT));
    uint32_t phase = 0;                                      // bit p: parity of s_bar[p]

    const double beta = __ldcg(s.beta + rep);
    const double cut_span = 20.0 / beta;                    // CPU_PIM.cpp:234
    int64_t E = __ldcg((const long long *)s.E + rep), bestE = __ldcg((const long long *)s.bestE + rep);
    unsigned long long accepts = 0;
    const uint32_t k0 = (uint32_t)s.seed, k1 = (uint32_t)(s.seed >> 32);
    const int K = (n + BT - 1) / BT;                         // weights per thread (<= 4)
    const int nvec = npad / VEC;
    bool failed = false;
    int upd = 0;                                             // update counter (buffer parity)

    for (int sw = 0; sw < s.spe && !failed; ++sw) {
        const uint32_t sweep = (uint32_t)(e * s.spe + sw);
        // r of every update of this sweep (:212), one Philox block each, drawn by all threads up
        // front; the picks read them after their barriers (the last pick of the previous sweep
        // read its r before its final barrier)
        for (int q = tid; q < n; q += BT) {
            if (s.replay_r) {   // a replay with the caller's uniforms
                s_r[q] = __ldcg(s.replay_r + (size_t)sweep * n + q);
                continue;
            }
            uint32_t w0, w1;
            philox_2words((uint32_t)q, sweep, (uint32_t)l, (uint32_t)g, k0, k1, w0, w1);
            s_r[q] = canonical53(w0, w1);
        }
        for (int i = 0; i < n; ++i, ++upd) {
            const int p = upd & 1;
            if constexpr (CL > 1) {
                if (tid == 0) mbar_arrive_expect_tx(smem_u32(&s_bar[p]), tx_bytes);
            }
            const int a = s_phi[i];
            const int inext = (i + 1 == n) ? 0 : i + 1;
            const int32_t *Di = s_Drow + p * rpc;            // D[i][own rows]
            const int32_t *DTi = SYM ? Di : s_DTrow + p * rpc;
            const int32_t *Fa = s_Frow + p * npad;           // F[a][*]
            const int32_t *FTa = SYM ? Fa : s_FTrow + p * npad;
            {   // rows of the next update (its facility assumes this update keeps phi)
                const int an = s_phi[inext];
                prefetch_rows<SYM>(tid, BT, nDc, s.D + (size_t)inext * ldm + row0,
                                   s.DT + (size_t)inext * ldm + row0, s_Drow + (p ^ 1) * rpc,
                                   s_DTrow + (p ^ 1) * rpc, nFc, s.F + (size_t)an * ldm,
                                   s.FT + (size_t)an * ldm, s_Frow + (p ^ 1) * npad,
                                   s_FTrow + (p ^ 1) * npad);
            }

            // ---- 1. delta halves: B from the rows this CTA owns, A from row i's owner
            int owner = 0;                                   // i / rpc without a division
#pragma unroll
            for (int r = 1; r < CL; ++r) owner += i >= r * rpc;
            const int32_t Dii = s_Dd[i], Faa = s_Fd[a];
            IT Iia = 0;
            const IT *Ii = sI + (size_t)(i - owner * rpc) * lds;
            if (owner == rank) Iia = Ii[a];
            for (int jj = tid; jj < rows; jj += BT) {
                const int j = row0 + jj;
                const int b = s_phi[j];
                const IT *Ij = sI + (size_t)jj * lds;
                const U dd = (U)(IT)Dii + (U)(IT)s_Dd[j] - (U)(IT)Di[jj] - (U)(IT)DTi[jj];
                const U ff = (U)(IT)Faa + (U)(IT)s_Fd[b] - (U)(IT)Fa[b] - (U)(IT)FTa[b];
                const U Bv = (U)Ij[a] - (U)Ij[b] - dd * ff;
                if constexpr (CL == 1) {
                    s_A[p * npad + b] = (IT)(Bv + (U)Ii[b] - (U)Iia);
                } else {
#pragma unroll
                    for (int r = 0; r < CL; ++r)
                        st_async(B_at[r] + (uint32_t)((p * npad + b) * sizeof(IT)), (IT)Bv, bar_at[r] + p * 8);
                }
            }
            if constexpr (CL > 1) {
                if (owner == rank) {
                    for (int c4 = tid; c4 < npad / VEC; c4 += BT) {
                        Vec<IT> v = *reinterpret_cast<const Vec<IT> *>(Ii + c4 * VEC);
#pragma unroll
                        for (int q = 0; q < VEC; ++q) v.v[q] = (IT)((U)v.v[q] - (U)Iia);
#pragma unroll
                        for (int r = 0; r < CL; ++r)
                            st_async16(A_at[r] + (uint32_t)((p * npad + c4 * VEC) * sizeof(IT)), v,
                                       bar_at[r] + p * 8);
                    }
                }
            }

            // ---- 2. all deltas present: max, heat-bath weights, prefix sum, threshold pick
            bool timeout = false;
            if constexpr (CL == 1) {
                G.sync();
            } else {
                timeout = !mbar_wait_bounded(smem_u32(&s_bar[p]), (phase >> p) & 1u, kWaitLimitNs);
                phase ^= 1u << p;
            }
            const int b0 = tid * K;
            IT d[4];
            double x[4];
            IT lmax = 0;                                     // max starts at 0 (:208)
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                d[k] = 0;
                x[k] = 0.0;
                if (k < K && b0 + k < n) {
                    const int b = b0 + k;
                    d[k] = (CL == 1) ? s_A[p * npad + b]
                                     : (IT)((U)s_A[p * npad + b] + (U)s_B[p * npad + b]);
                    lmax = d[k] > lmax ? d[k] : lmax;
                }
            }
            lmax = warp_max(lmax);
            if (lane == 0) s_red[warp] = lmax;
            if (G.sync_or(timeout)) {                 // S_max
                if (tid == 0) atomicOr(s.error, kErrTimeout);
                failed = true;
                break;
            }
            if (tid == 0) s_misc[0] = 0x7fffffff;
            // the weights do not depend on the maximum: formed while it is read
            const IT M = block_max(s_red, nwarps, lane);
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k < K && b0 + k < n) x[k] = exp2(__dmul_rn(beta, (double)d[k]));
            const long long cut = cutoff_trunc(__dsub_rn((double)M, cut_span));   // :234-235
            double pre[4];
            double local = 0.0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (k < K && (long long)d[k] > cut && b0 + k < n) local = __dadd_rn(local, x[k]);
                pre[k] = local;
            }
            double incl = local;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl = __dadd_rn(incl, y);
            }
            double excl = __shfl_up_sync(0xffffffffu, incl, 1);
            if (lane == 0) excl = 0.0;
            if (lane == 31) s_wsum[warp] = incl;
            G.sync();                                 // S_scan
            double base, total;
            weight_totals(s_wsum, nwarps, warp, base, total);
            const double target = __dmul_rn(s_r[i], total);     // :247
            const double X = __dadd_rn(base, excl);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (k < K && b0 + k < n) {
                    if (__dadd_rn(X, pre[k]) >= target) {   // :251
                        atomicMin(&s_misc[0], b0 + k);
                        break;
                    }
                }
            }
            cp_async_wait_all();                             // next update's rows have landed
            G.sync();                                 // S_pick
            const int bs = s_misc[0];
            if (bs >= n || bs == a) continue;                // no move / self move (:252)

            // ---- 3. accepted swap: i gets facility bs, j = phiinv(bs) gets a
            const int j = s_inv[bs];
            const IT dEsel = (CL == 1) ? s_A[p * npad + bs]
                                       : (IT)((U)s_A[p * npad + bs] + (U)s_B[p * npad + bs]);
            prefetch_rows<SYM>(tid, BT, nDc, s.D + (size_t)j * ldm + row0, s.DT + (size_t)j * ldm + row0,
                               s_Dj, s_DTj, nFc, s.F + (size_t)bs * ldm, s.FT + (size_t)bs * ldm,
                               s_Fb, s_FTb);
            cp_async_wait_all();
            // the row factors of the rank-2 update, each computed by the thread that fetched
            // its 16-byte chunk of row j (prefetch_rows' chunk order), so no extra barrier
            for (int q = tid; q < (SYM ? nDc : 2 * nDc + nFc); q += BT) {
                if (q < nDc) {
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        const int k = 4 * q + r;
                        const U d = (U)(IT)s_Dj[k] - (U)(IT)Di[k];
                        if constexpr (SYM) s_u1[k] = (IT)(2u * d);
                        else s_u2[k] = (IT)d;
                    }
                } else if (!SYM && q >= nDc + nFc) {
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        const int k = 4 * (q - nDc - nFc) + r;
                        s_u1[k] = (IT)((U)(IT)s_DTj[k] - (U)(IT)DTi[k]);
                    }
                }
            }
            G.sync();                                 // S4: rows j / bs and the row factors in shared memory
            if (tid == 0) {
                s_phi[i] = bs;                               // :257-261
                s_inv[bs] = i;
                s_phi[j] = a;
                s_inv[a] = j;
            }
            if (j == inext) {   // the next location's facility became a: its F rows are Fa/FTa
                for (int c = tid; c < npad; c += BT) {
                    s_Frow[(p ^ 1) * npad + c] = Fa[c];
                    if constexpr (!SYM) s_FTrow[(p ^ 1) * npad + c] = FTa[c];
                }
            }
            E -= (int64_t)dEsel;                             // :256
            ++accepts;
            if (E < bestE) {                                 // :271-272
                bestE = E;
                if (tid == 0) {
                    s_misc[1] = upd;
                    if constexpr (GP) {
                        if (E < s.ev.goal_print && rank == 0) s_misc[3] = goal_print_claim(s.ev, g, l, e, E);
                    }
                }
            }
            // I[k][c] += (D[k][j]-D[k][i])(F[c][b]-F[c][a]) + (D[j][k]-D[i][k])(F[b][c]-F[a][c])
            for (int cv = tid % nvec, k0r = tid / nvec, kstep = max(1, BT / nvec);
                 cv < nvec; cv += (BT >= nvec ? nvec : BT)) {
                if (BT >= nvec && k0r >= kstep) break;
                Vec<IT> v1, v2;
#pragma unroll
                for (int q = 0; q < VEC; ++q) {
                    const int c = cv * VEC + q;
                    if constexpr (SYM) {
                        v1.v[q] = (IT)((U)(IT)s_Fb[c] - (U)(IT)Fa[c]);
                    } else {
                        v1.v[q] = (IT)((U)(IT)s_FTb[c] - (U)(IT)FTa[c]);
                        v2.v[q] = (IT)((U)(IT)s_Fb[c] - (U)(IT)Fa[c]);
                    }
                }
                const int kfirst = (BT >= nvec) ? k0r : 0;
                const int kinc = (BT >= nvec) ? kstep : 1;
                auto upd_row = [&](int k, Vec<IT> &x) {
                    const U u1 = (U)s_u1[k];
                    if constexpr (SYM) {
#pragma unroll
                        for (int q = 0; q < VEC; ++q) x.v[q] = (IT)((U)x.v[q] + u1 * (U)v1.v[q]);
                    } else {
                        const U u2 = (U)s_u2[k];
#pragma unroll
                        for (int q = 0; q < VEC; ++q)
                            x.v[q] = (IT)((U)x.v[q] + u1 * (U)v1.v[q] + u2 * (U)v2.v[q]);
                    }
                };
                // rows in batches: the loads of a batch are in flight together
                constexpr int RB = sizeof(IT) == 8 ? 2 : 8;
                int k = kfirst;
                for (; k + (RB - 1) * kinc < rows; k += RB * kinc) {
                    Vec<IT> x[RB];
#pragma unroll
                    for (int m = 0; m < RB; ++m)
                        x[m] = *reinterpret_cast<const Vec<IT> *>(sI + (size_t)(k + m * kinc) * lds + cv * VEC);
#pragma unroll
                    for (int m = 0; m < RB; ++m) upd_row(k + m * kinc, x[m]);
#pragma unroll
                    for (int m = 0; m < RB; ++m)
                        *reinterpret_cast<Vec<IT> *>(sI + (size_t)(k + m * kinc) * lds + cv * VEC) = x[m];
                }
                for (; k < rows; k += kinc) {
                    Vec<IT> *dst = reinterpret_cast<Vec<IT> *>(sI + (size_t)k * lds + cv * VEC);
                    Vec<IT> x = *dst;
                    upd_row(k, x);
                    *dst = x;
                }
            }
            G.sync();                                 // S5: new rows and phi visible
            if (s_misc[1] == upd) {
                for (int q = tid; q < n; q += BT) s_bphi[q] = s_phi[q];
                if constexpr (GP) {
                    if (E < s.ev.goal_print && rank == 0) {
                        const int slot = s_misc[3];
                        if (slot >= 0)
                            for (int q = tid; q < n; q += BT) s.ev.perm[(size_t)slot * n + q] = s_phi[q];
                    }
                }
            }
        }
    }

    // ---- store the replica, then the last replica of the group runs the exchange
    cp_async_wait_all();
    cluster_sync<CL>(G);   // all deltas exchanged; no CTA writes into another any more
    if constexpr (CL > 1) {
        if (tid == 0) {
            mbar_inval(smem_u32(&s_bar[0]));
            mbar_inval(smem_u32(&s_bar[1]));
        }
    }
    if (failed) return false;
    {
        IT *gI = reinterpret_cast<IT *>(s.I) + ((size_t)rep * n + row0) * s.ldg;
        const int nvg = s.ldg / VEC;
        for (int idx = tid; idx < rows * nvg; idx += BT) {
            const int k = idx / nvg, v = idx - k * nvg;
            *reinterpret_cast<Vec<IT> *>(gI + (size_t)k * s.ldg + v * VEC) =
                *reinterpret_cast<const Vec<IT> *>(sI + (size_t)k * lds + v * VEC);
        }
    }
    if (rank == 0) {
        int32_t *gphi = s.phi + (size_t)rep * n;
        for (int q = tid; q < n; q += BT) gphi[q] = s_phi[q];
        if (s_misc[1] >= 0) {
            int32_t *gb = s.best_phi + (size_t)rep * n;
            for (int q = tid; q < n; q += BT) gb[q] = s_bphi[q];
        }
        if (tid == 0) {
            s.E[rep] = E;
            s.bestE[rep] = bestE;
            s.accepts[rep] = __ldcg(s.accepts + rep) + accepts;
        }
    }
    __threadfence();   // this thread's stores reach L2 before the worker reports the epoch done
    return true;
}

// ---- tcgen05: the 5th-generation tensor cores.  Operands in shared memory, named by matrix
// descriptors; fp32 accumulators in tensor memory (TMEM: 128 lanes x 512 columns of 32 bits
// per SM, lane m = row m of an M = 128 product); one thread issues, an mbarrier reports the
// completion.

// Shared-memory matrix descriptor of an fp16 operand stored MN-major without swizzle: core
// matrices of 8 K-rows x 16 bytes (8 consecutive M or N entries), 128 contiguous bytes each;
// kstride = bytes between core matrices adjacent in K (the leading byte offset), mnstride =
// bytes between core matrices adjacent in M / N (the stride byte offset).  Bits: start
// address >> 4 [0, 14), leading offset >> 4 [16, 30), stride offset >> 4 [32, 46), descriptor
// version 1 [46, 48), base offset 0, layout type 0 (no swizzle) [61, 64).
__device__ __forceinline__ uint64_t umma_desc_mn(uint32_t saddr, uint32_t kstride, uint32_t mnstride) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((kstride >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((mnstride >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of tcgen05.mma kind::f16 with fp16 A and B, both MN-major, and an
// fp32 accumulator, M x N: D format [4, 6) = 1 (f32), A / B format [7, 10) / [10, 13) = 0
// (f16), A / B major [15] / [16] = 1 (MN), N >> 3 [17, 23), M >> 4 [24, 29).
__host__ __device__ constexpr uint32_t umma_idesc_f16_mn(int M, int N) {
    return (1u << 4) | (1u << 15) | (1u << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Allocation of ncols tensor-memory columns (a power of two >= 32) by one whole warp; the
// address is written to shared memory at dst.
__device__ __forceinline__ void tmem_alloc(uint32_t dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// Orders this thread's tcgen05 operations before (after) a following (preceding) barrier.
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Makes this thread's shared-memory stores visible to the tensor cores' (async-proxy) reads.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D (TMEM) = A B (+ D when accumulate), M x N x 16, one thread.
__device__ __forceinline__ void umma_f16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}
// The mbarrier at bar gets one arrival when every tcgen05.mma this thread issued has completed.
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}
// 16 consecutive 32-bit columns of the warp's 32 TMEM lanes (thread t: lane base + t); the
// values are valid after tmem_wait_ld.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
        "%13, %14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Eight small integers (exact in fp16) as eight fp16 in one 16-byte word, element 0 first.
template <class T>
__device__ __forceinline__ uint4 pack_f16x8(T a, T b, T c, T d, T e, T f, T g, T h) {
    const __half2 h0 = __floats2half2_rn((float)a, (float)b), h1 = __floats2half2_rn((float)c, (float)d);
    const __half2 h2 = __floats2half2_rn((float)e, (float)f), h3 = __floats2half2_rn((float)g, (float)h);
    uint4 r;
    memcpy(&r.x, &h0, 4);
    memcpy(&r.y, &h1, 4);
    memcpy(&r.z, &h2, 4);
    memcpy(&r.w, &h3, 4);
    return r;
}

// Shared-memory layout of the binary-flow epoch (replica_epoch_bin): the instance itself is
// resident next to the force-matrix rows, D as int16 columns of this CTA's rows and F as bit
// rows, so no update waits for a row from L2.
constexpr int kBinLog = 16;   // accepted swaps the binary-flow epoch keeps before rewriting its rows
// The staged A operand of the tensor-core rewrite: 16 groups of 8 rows x 2 core matrices of
// 8 log entries x 8 rows x 2 bytes.
constexpr int kBinTcA = 16 * 256;

//   inst = false: the replica's own section only (no Ds / Fb), for two replicas of one
//   instance that share one copy of the instance tables (BinPairLayout).
//   tcr = true: the rows are rewritten on the tcgen05 tensor cores (replica_epoch_bin): the log
//   region [LU, V8 end) also holds, once the log is full, its entries restaged as fp16 MN-major
//   core matrices (A: 128 rows x 16 entries, 4 KB; B: columns rounded up to 16 x 16 entries,
//   32 B per column), and `tc` holds the MMA's mbarrier and the tensor-memory address.
struct BinLayout {
    size_t I, phi, inv, bphi, Dd, A, B, Ds, Fb, LU, V8, red, wsum, r, misc, bar, tc, total;
    __host__ __device__ BinLayout(int n, int rpc, int lds, int cluster, bool inst = true, bool tcr = false) {
        const size_t npad = (size_t)((n + 3) & ~3), rp = (size_t)rpc, nw = (size_t)((n + 31) / 32);
        const size_t ni = inst ? (size_t)n : 0;
        size_t o = 0;
        I = o;     o = align16(o + rp * lds * 4);
        phi = o;   o = align16(o + npad * 4);
        inv = o;   o = align16(o + npad * 4);
        bphi = o;  o = align16(o + npad * 4);
        Dd = o;    o = align16(o + npad * 4);
        A = o;     o = align16(o + 2 * npad * 4);
        B = o;     o = align16(o + (cluster > 1 ? 2 * npad * 4 : 0));
        Ds = o;    o = align16(o + ni * rp * 2);   // Ds[r][k] = D[r][row0 + k]
        Fb = o;    o = align16(o + ni * nw * 4);   // bit b % 32 of Fb[a][b / 32] = F[a][b]
        LU = o;    o = align16(o + (size_t)kBinLog * rp * 4);   // LU[p][k] = 2 (D[k][j_p] - D[k][i_p])
        V8 = o;    o = align16(o + (size_t)kBinLog * npad);     // V8[p][c] = F[b_p][c] - F[a_p][c]
        if (tcr) {   // room for the staged operands
            const size_t staged = (size_t)kBinTcA + (size_t)((n + 15) & ~15) * 32;
            if (o - LU < staged) o = LU + staged;
        }
        red = o;   o = align16(o + kMaxWarps * 8);
        wsum = o;  o = align16(o + kMaxWarps * sizeof(double));
        r = o;     o = align16(o + npad * sizeof(double));   // r of each update of a sweep
        misc = o;  o = align16(o + 4 * sizeof(int));
        bar = o;   o = align16(o + 2 * sizeof(unsigned long long));
        tc = o;    o = align16(o + (tcr ? 16 : 0));
        total = o;
    }
};

// Two replicas of one instance per CTA (the paired binary-flow epoch): the instance tables
// Ds / Fb once, then one replica section per replica.  Each replica is run by half of the CTA's
// warps with its own named barrier, so the two update chains interleave on the SM and each
// hides the other's barrier and shared-memory latency.
struct BinPairLayout {
    size_t Ds, Fb, rep[2], total;
    __host__ __device__ BinPairLayout(int n, int rpc, int lds, int cluster) {
        const size_t rp = (size_t)rpc, nw = (size_t)((n + 31) / 32);
        // each section also holds the exchange scratch once its replica's epoch is done
        const size_t slice = align16(max(BinLayout(n, rpc, lds, cluster, false).total, kExchangeScratchBytes));
        size_t o = 0;
        Ds = o;     o = align16(o + (size_t)n * rp * 2);
        Fb = o;     o = align16(o + (size_t)n * nw * 4);
        rep[0] = o; o += slice;
        rep[1] = o; o += slice;
        total = o;
    }
};

size_t epoch_smem_bytes_bin(int n, int rpc, int lds, int cluster, bool tcr) {
    return BinLayout(n, rpc, lds, cluster, true, tcr).total;
}

size_t epoch_smem_bytes_bin_pair(int n, int rpc, int lds, int cluster) {
    return BinPairLayout(n, rpc, lds, cluster).total;
}

// The binary-flow instance tables of cluster rank `rank` in shared memory: Ds[r][k] =
// D[r][row0 + k] for the CTA's rows (int16) and F as bit rows.  Run by threads tid = 0..BT-1.
__device__ __forceinline__ void load_bin_instance(const SolveDev &s, int rank, int tid, int BT, int lane,
                                                  int warp, int nwarps, int16_t *s_Ds, uint32_t *s_Fb) {
    const int n = s.n, rpc = s.rpc, ldm = s.ldm, nw = (n + 31) / 32;
    const int row0 = rank * rpc;
    const int rows = max(0, min(rpc, n - row0));
    for (int idx = tid; idx < n * rows; idx += BT) {
        const int r = idx / rows, k = idx - r * rows;
        s_Ds[(size_t)r * rpc + k] = (int16_t)__ldcg(s.D + (size_t)r * ldm + row0 + k);
    }
    for (int widx = warp; widx < n * nw; widx += nwarps) {
        const int r = widx / nw, w = widx - r * nw, b = 32 * w + lane;
        const bool one = b < n && __ldcg(s.F + (size_t)r * ldm + b) != 0;
        const unsigned bits = __ballot_sync(0xffffffffu, one);
        if (lane == 0) s_Fb[widx] = bits;
    }
}

// One epoch of replica rep for a symmetric instance whose flows are 0 / 1 and whose distances
// fit in int16 (int32 force matrix): replica_epoch with the instance resident in shared memory.
// Every delta, weight and update is the same integer / fp64 computation as replica_epoch's:
// dd = Dii + Djj - 2 Dij, ff = Faa + Fbb - 2 Fab, and the rank-2 update
// I[k][c] += 2 (Djk - Dik)(Fbc - Fac) (CPU_PIM.cpp:220-232, :262-268 with D = Dᵀ, F = Fᵀ).
//   Ds_shared / Fb_shared (both or neither): the instance tables, already loaded by the caller
//   into shared memory that another replica of the same instance uses too; smem then holds
//   only this replica's section (BinLayout with inst = false).
template <int CL>
__device__ bool replica_epoch_bin(const SolveDev &s, int rep, int rank, int e, const Grp &G,
                                  unsigned char *smem, int16_t *Ds_shared = nullptr,
                                  uint32_t *Fb_shared = nullptr) {
    using IT = int32_t;
    using U = uint32_t;
    constexpr int VEC = 4;
    const int n = s.n;
    const int tid = G.tid, BT = G.BT, lane = G.lane, warp = G.warp, nwarps = G.nwarps;
    const int g = rep / s.R, l = rep - g * s.R;
    const int rpc = s.rpc, lds = s.lds, ldm = s.ldm;
    const int row0 = rank * rpc;
    const int rows = max(0, min(rpc, n - row0));
    const int npad = (n + 3) & ~3;
    const int nw = (n + 31) / 32;
    const bool own_inst = Ds_shared == nullptr;
    const bool tcr = own_inst && s.bin_tc != 0;             // rows rewritten on the tensor cores
    const BinLayout L(n, rpc, lds, CL, own_inst, tcr);
    IT *sI = reinterpret_cast<IT *>(smem + L.I);
    int32_t *s_phi = reinterpret_cast<int32_t *>(smem + L.phi);
    int32_t *s_inv = reinterpret_cast<int32_t *>(smem + L.inv);
    int32_t *s_bphi = reinterpret_cast<int32_t *>(smem + L.bphi);
    int32_t *s_Dd = reinterpret_cast<int32_t *>(smem + L.Dd);
    IT *s_A = reinterpret_cast<IT *>(smem + L.A);
    IT *s_B = reinterpret_cast<IT *>(smem + L.B);
    int16_t *s_Ds = own_inst ? reinterpret_cast<int16_t *>(smem + L.Ds) : Ds_shared;
    uint32_t *s_Fb = own_inst ? reinterpret_cast<uint32_t *>(smem + L.Fb) : Fb_shared;
    float *s_LU = reinterpret_cast<float *>(smem + L.LU);
    int8_t *s_V8 = reinterpret_cast<int8_t *>(smem + L.V8);
    IT *s_red = reinterpret_cast<IT *>(smem + L.red);
    double *s_wsum = reinterpret_cast<double *>(smem + L.wsum);
    double *s_r = reinterpret_cast<double *>(smem + L.r);
    int *s_misc = reinterpret_cast<int *>(smem + L.misc);   // [0] pick key, [1] improved-at
    unsigned long long *s_bar = reinterpret_cast<unsigned long long *>(smem + L.bar);
    auto fbit = [&](int a, int b) -> int { return (int)((s_Fb[a * nw + (b >> 5)] >> (b & 31)) & 1u); };

    const int tcn = (n + 15) & ~15;                          // the rewrite MMA's N
    const uint32_t tcols = tcn <= 32 ? 32u : (tcn <= 64 ? 64u : (tcn <= 128 ? 128u : 256u));
    const uint32_t tc_bar = smem_u32(smem + L.tc);
    uint32_t tmem = 0, tc_phase = 0;
    bool tc_dead = false;                                    // a wait for the rewrite MMA gave up

    // ---- load the replica and the instance
    {
        const IT *gI = reinterpret_cast<const IT *>(s.I) + ((size_t)rep * n + row0) * s.ldg;
        const int nvg = s.ldg / VEC;
        for (int idx = tid; idx < rows * nvg; idx += BT) {
            const int k = idx / nvg, v = idx - k * nvg;
            const int4 w = __ldcg(reinterpret_cast<const int4 *>(gI + (size_t)k * s.ldg + v * VEC));
            *reinterpret_cast<int4 *>(sI + (size_t)k * lds + v * VEC) = w;
        }
        const int32_t *gphi = s.phi + (size_t)rep * n;
        for (int q = tid; q < npad; q += BT) {
            int p = q < n ? __ldcg(gphi + q) : 0;
            if ((unsigned)p >= (unsigned)n) {
                atomicOr(s.error, kErrBadPerm);
                p = 0;
            }
            s_phi[q] = p;
            s_bphi[q] = p;
            s_inv[q] = 0;
            s_Dd[q] = q < n ? __ldcg(s.Ddiag + q) : 0;
        }
        if (own_inst) load_bin_instance(s, rank, tid, BT, lane, warp, nwarps, s_Ds, s_Fb);
        if (tid == 0) {
            s_misc[0] = 0x7fffffff;
            s_misc[1] = -1;
            if constexpr (CL > 1) {
                mbar_init(smem_u32(&s_bar[0]), 1);
                mbar_init(smem_u32(&s_bar[1]), 1);
                mbar_fence_init();
            }
        }
        if (tcr) {
            // the rewrite's sums live in tcols tensor-memory columns (warp 0 allocates them; the
            // host caps the CTAs per SM at 512 / tcols, so the allocation does not wait), and
            // its MMA completes on one mbarrier
            __syncwarp();
            if (warp == 0) tmem_alloc(smem_u32(smem + L.tc + 8), tcols);
            if (tid == 0) {
                mbar_init(tc_bar, 1);
                mbar_fence_init();
            }
            tc_fence_before();
        }
        G.sync();
        if (tcr) {
            tc_fence_after();
            tmem = *reinterpret_cast<volatile uint32_t *>(smem + L.tc + 8);
        }
    }
    for (int q = tid; q < n; q += BT) s_inv[s_phi[q]] = q;
    cluster_sync<CL>(G);

    uint32_t A_at[CL], B_at[CL], bar_at[CL];
    if constexpr (CL > 1) {
#pragma unroll
        for (int r = 0; r < CL; ++r) {
            A_at[r] = cluster_addr(smem_u32(s_A), r);
            B_at[r] = cluster_addr(smem_u32(s_B), r);
            bar_at[r] = cluster_addr(smem_u32(s_bar), r);
        }
    }
    const uint32_t tx_bytes = (uint32_t)((npad + n) * sizeof(IT));
    uint32_t phase = 0;

    const double beta = __ldcg(s.beta + rep);
    const double cut_span = 20.0 / beta;                    // CPU_PIM.cpp:234
    int64_t E = __ldcg((const long long *)s.E + rep), bestE = __ldcg((const long long *)s.bestE + rep);
    unsigned long long accepts = 0;
    const uint32_t k0 = (uint32_t)s.seed, k1 = (uint32_t)(s.seed >> 32);
    const int K = (n + BT - 1) / BT;                         // weights per thread (<= 4)
    const int nvec = npad / VEC;
    const int act = s.act;
    bool failed = false;
    int upd = 0;
    // Deferred force updates (not for clique flows): an accepted swap p is logged as the row
    // factors LU[p][k] = 2 (D[k][j_p] - D[k][i_p]) of this CTA's rows and the column factors
    // V8[p][c] = F[b_p][c] - F[a_p][c] (int8); a force entry is then
    // I[k][c] + sum_p LU[p][k] V8[p][c].  The sums are formed in binary32, which is exact here:
    // |LU| <= 2^17 (int16 distances), |V8| <= 1, at most kBinLog = 16 terms, so every partial
    // sum (also of the corrections below, |weight| <= 2) stays below 2^24.  Each
    // update corrects the entries it reads; every kBinLog swaps (and at the end of the epoch)
    // the rows are rewritten once for all of them.  Integer sums in any order: exact.
    const bool lazy = act == 0;
    int m = 0;                                               // pending swaps (same in all CTAs)
    // The rewrite on the tcgen05 tensor cores (tcr): I[k][c] += sum_p LU[p][k] V8[p][c] as one
    // M = 128, N = tcn, K = 16 MMA with fp16 operands and fp32 sums in tensor memory.  Exact:
    // the host enables it only where |LU| <= 2048 (twice the instance's distance range at
    // most 1024), |V8| <= 1, and 16 terms keep every sum below 2^24.  The log entries are
    // restaged in place (every thread reads its chunks, a barrier, then writes them) as fp16
    // MN-major core matrices without swizzle: 8 rows (or columns) x 8 entries, 16 bytes per
    // entry, 128 bytes each; 128 bytes between the two core matrices of a group along the
    // entries (LBO), 256 bytes between groups of 8 rows or columns (SBO).  Entries past m are
    // zero, rows past rpc and columns past npad too.  Warp w reads back tensor-memory lanes
    // 32 (w % 4) .. + 31 (its rows), 16 columns at a time, and adds the sums to the rows.
    auto flush_tc = [&]() {
        constexpr int kChunks = 6;                            // (256 + 512) chunks / 128 threads
        const int nA = 16 * kBinLog, nB = (tcn / 8) * kBinLog;
        uint4 v[kChunks];
#pragma unroll
        for (int t = 0; t < kChunks; ++t) {
            const int c = tid + t * BT;
            uint4 w = make_uint4(0u, 0u, 0u, 0u);
            if (c < nA) {
                const int p = c >> 4, g = c & 15;             // log entry, group of 8 rows
                if (p < m && 8 * g < rpc) {
                    const float *lu = s_LU + (size_t)p * rpc + 8 * g;
                    const float4 f0 = *reinterpret_cast<const float4 *>(lu);
                    const float4 f1 = (8 * g + 4 < rpc) ? *reinterpret_cast<const float4 *>(lu + 4)
                                                        : make_float4(0.f, 0.f, 0.f, 0.f);
                    w = pack_f16x8(f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w);
                }
            } else if (c < nA + nB) {
                const int c2 = c - nA, p = c2 & 15, cg = c2 >> 4;   // log entry, group of 8 columns
                if (p < m && 8 * cg < npad) {
                    const int8_t *v8 = s_V8 + (size_t)p * npad + 8 * cg;
                    const char4 b0 = *reinterpret_cast<const char4 *>(v8);
                    const char4 b1 = (8 * cg + 4 < npad) ? *reinterpret_cast<const char4 *>(v8 + 4)
                                                         : make_char4(0, 0, 0, 0);
                    w = pack_f16x8(b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w);
                }
            }
            v[t] = w;
        }
        G.sync();                                             // every log entry read
#pragma unroll
        for (int t = 0; t < kChunks; ++t) {
            const int c = tid + t * BT;
            if (c < nA) {
                const int p = c >> 4, g = c & 15;
                *reinterpret_cast<uint4 *>(smem + L.LU + (size_t)g * 256 + (p >> 3) * 128 + (p & 7) * 16) = v[t];
            } else if (c < nA + nB) {
                const int c2 = c - nA, p = c2 & 15, cg = c2 >> 4;
                *reinterpret_cast<uint4 *>(smem + L.LU + kBinTcA + (size_t)cg * 256 + (p >> 3) * 128 + (p & 7) * 16) =
                    v[t];
            }
        }
        fence_async_smem();
        G.sync();                                             // the operands are staged
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a = smem_u32(smem + L.LU);
            umma_f16(tmem, umma_desc_mn(a, 128u, 256u), umma_desc_mn(a + kBinTcA, 128u, 256u),
                     umma_idesc_f16_mn(128, tcn), false);
            umma_commit(tc_bar);
        }
        const bool gave_up = !mbar_wait_bounded(tc_bar, tc_phase, kWaitLimitNs);
        tc_phase ^= 1u;
        if (G.sync_or(gave_up)) {
            if (tid == 0) atomicOr(s.error, kErrTimeout);
            tc_dead = true;
            failed = true;
            return;
        }
        tc_fence_after();
        const int quad = warp & 3, r = 32 * quad + lane;
        for (int cb = warp >> 2; 16 * cb < tcn; cb += nwarps >> 2) {
            uint32_t acc[16];
            tmem_ld16(tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)(16 * cb), acc);
            tmem_wait_ld();
            if (r < rows) {
                IT *dst = sI + (size_t)r * lds + 16 * cb;
                if (16 * cb + 16 <= npad) {
#pragma unroll
                    for (int q4 = 0; q4 < 4; ++q4) {
                        int4 x = *reinterpret_cast<const int4 *>(dst + 4 * q4);
                        x.x = (int)((U)x.x + (U)__float2int_rn(__uint_as_float(acc[4 * q4 + 0])));
                        x.y = (int)((U)x.y + (U)__float2int_rn(__uint_as_float(acc[4 * q4 + 1])));
                        x.z = (int)((U)x.z + (U)__float2int_rn(__uint_as_float(acc[4 * q4 + 2])));
                        x.w = (int)((U)x.w + (U)__float2int_rn(__uint_as_float(acc[4 * q4 + 3])));
                        *reinterpret_cast<int4 *>(dst + 4 * q4) = x;
                    }
                } else {
#pragma unroll
                    for (int t = 0; t < 16; ++t)
                        if (16 * cb + t < npad) dst[t] = (IT)((U)dst[t] + (U)__float2int_rn(__uint_as_float(acc[t])));
                }
            }
        }
        tc_fence_before();                                    // before the next rewrite's MMA
    };
    auto flush = [&]() {
        if (tcr) {
            flush_tc();
            return;
        }
        // rows in blocks of 8 consecutive rows x 4 columns per thread
        constexpr int RT = 8;
        const int ngroups = max(1, BT / nvec);               // row-block groups in flight
        for (int cv = tid % nvec, grp = tid / nvec; cv < nvec; cv += (BT >= nvec ? nvec : BT)) {
            if (BT >= nvec && grp >= ngroups) break;
            const int c0 = cv * VEC;
            const int gfirst = (BT >= nvec) ? grp : 0, ginc = (BT >= nvec) ? ngroups : 1;
            for (int kb = gfirst * RT; kb < rows; kb += ginc * RT) {
                float acc[RT][VEC];
#pragma unroll
                for (int r = 0; r < RT; ++r)
#pragma unroll
                    for (int q = 0; q < VEC; ++q) acc[r][q] = 0.0f;
                for (int p = 0; p < m; ++p) {
                    const char4 v4 = *reinterpret_cast<const char4 *>(s_V8 + (size_t)p * npad + c0);
                    const float v[VEC] = {(float)v4.x, (float)v4.y, (float)v4.z, (float)v4.w};
                    // LU rows are rpc long (a multiple of 4) and 16-byte aligned; rows past `rows`
                    // hold zeros and are never written back
                    const float4 l0 = *reinterpret_cast<const float4 *>(s_LU + (size_t)p * rpc + kb);
                    const float4 l1 = (kb + 4 < rpc) ? *reinterpret_cast<const float4 *>(s_LU + (size_t)p * rpc + kb + 4)
                                                     : make_float4(0.f, 0.f, 0.f, 0.f);
                    const float u[RT] = {l0.x, l0.y, l0.z, l0.w, l1.x, l1.y, l1.z, l1.w};
#pragma unroll
                    for (int r = 0; r < RT; ++r)
#pragma unroll
                        for (int q = 0; q < VEC; ++q) acc[r][q] = fmaf(u[r], v[q], acc[r][q]);
                }
#pragma unroll
                for (int r = 0; r < RT; ++r) {
                    if (kb + r < rows) {
                        Vec<IT> *dst = reinterpret_cast<Vec<IT> *>(sI + (size_t)(kb + r) * lds + c0);
                        Vec<IT> xv = *dst;
#pragma unroll
                        for (int q = 0; q < VEC; ++q) xv.v[q] = (IT)((U)xv.v[q] + (U)(int)acc[r][q]);
                        *dst = xv;
                    }
                }
            }
        }
    };

    // Facilities kept in registers across updates, so an update's first shared-memory loads
    // need no earlier one: a_nx = phi of the next update's location (read during an update,
    // set for its swap; -1: read it), and, when every thread holds at most one row of the CTA
    // (rows <= BT), bj = phi of the thread's own row, kept through every swap.
    const bool one_row = rows <= BT;
    int a_nx = -1;
    int bj = (one_row && tid < rows) ? s_phi[row0 + tid] : 0;
    for (int sw = 0; sw < s.spe && !failed; ++sw) {
        const uint32_t sweep = (uint32_t)(e * s.spe + sw);
        // r of every update of this sweep (:212), one Philox block each, drawn by all threads up
        // front; the picks read them after their barriers (the last pick of the previous sweep
        // read its r before its final barrier)
        for (int q = tid; q < n; q += BT) {
            if (s.replay_r) {   // a replay with the caller's uniforms
                s_r[q] = __ldcg(s.replay_r + (size_t)sweep * n + q);
                continue;
            }
            uint32_t w0, w1;
            philox_2words((uint32_t)q, sweep, (uint32_t)l, (uint32_t)g, k0, k1, w0, w1);
            s_r[q] = canonical53(w0, w1);
        }
        for (int i = 0; i < n; ++i, ++upd) {
            const int p = upd & 1;
            if constexpr (CL > 1) {
                if (tid == 0) mbar_arrive_expect_tx(smem_u32(&s_bar[p]), tx_bytes);
            }
            const int a = a_nx >= 0 ? a_nx : s_phi[i];
            const int inext = i + 1 == n ? 0 : i + 1;
            // clique flows (act > 0): an inactive facility weighs the actives and one lumped
            // candidate b = act for all inactives (CPU_PIM_tai256c.cpp:236, :253-266)
            const bool inact = act > 0 && a >= act;
            const int ncand = inact ? act + 1 : n, npick = inact ? act : n;
            const int16_t *Di = s_Ds + (size_t)i * rpc;      // D[i][own rows]
            int owner = 0;                                   // i / rpc without a division
#pragma unroll
            for (int r = 1; r < CL; ++r) owner += i >= r * rpc;
            const int Dii = s_Dd[i], Faa = fbit(a, a);
            IT Iia = 0;
            const IT *Ii = sI + (size_t)(i - owner * rpc) * lds;
            if (owner == rank) Iia = Ii[a];
            for (int jj = tid; jj < rows; jj += BT) {
                const int j = row0 + jj;
                const int b = one_row ? bj : s_phi[j];
                const IT *Ij = sI + (size_t)jj * lds;
                const U dd = (U)Dii + (U)s_Dd[j] - 2u * (U)(IT)Di[jj];
                const U ff = (U)Faa + (U)fbit(b, b) - 2u * (U)fbit(a, b);
                U Bv = (U)Ij[a] - (U)Ij[b] - dd * ff;
                // pending swaps: I[j][a] - I[j][b] (and, with one CTA, I[i][b] - I[i][a]) as corrected
                float cf = 0.0f;
#pragma unroll 4
                for (int q = 0; q < m; ++q) {
                    const int8_t *v8 = s_V8 + (size_t)q * npad;
                    const float w = (float)((int)v8[a] - (int)v8[b]);
                    const float lu = (CL == 1) ? s_LU[q * rpc + jj] - s_LU[q * rpc + i] : s_LU[q * rpc + jj];
                    cf = fmaf(lu, w, cf);
                }
                Bv += (U)(int)cf;
                if constexpr (CL == 1) {
                    s_A[p * npad + b] = (IT)(Bv + (U)Ii[b] - (U)Iia);
                } else {
#pragma unroll
                    for (int r = 0; r < CL; ++r)
                        st_async(B_at[r] + (uint32_t)((p * npad + b) * sizeof(IT)), (IT)Bv, bar_at[r] + p * 8);
                }
            }
            if constexpr (CL > 1) {
                if (owner == rank) {
                    const int il = i - row0;
                    // on the threads after the B-half's when both fit, so the halves run side by side
                    const int aoff = (rows + nvec <= BT) ? rows : 0;
                    for (int c4 = tid - aoff; c4 >= 0 && c4 < nvec; c4 += BT) {
                        Vec<IT> v = *reinterpret_cast<const Vec<IT> *>(Ii + c4 * VEC);
#pragma unroll
                        for (int q = 0; q < VEC; ++q) v.v[q] = (IT)((U)v.v[q] - (U)Iia);
                        // pending swaps: I[i][c] - I[i][a] as corrected
                        const int c0 = c4 * VEC;
                        float cf[VEC] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll 4
                        for (int q2 = 0; q2 < m; ++q2) {
                            const int8_t *v8 = s_V8 + (size_t)q2 * npad;
                            const char4 v4 = *reinterpret_cast<const char4 *>(v8 + c0);
                            const int va = (int)v8[a];
                            const float lu = s_LU[q2 * rpc + il];
                            cf[0] = fmaf(lu, (float)((int)v4.x - va), cf[0]);
                            cf[1] = fmaf(lu, (float)((int)v4.y - va), cf[1]);
                            cf[2] = fmaf(lu, (float)((int)v4.z - va), cf[2]);
                            cf[3] = fmaf(lu, (float)((int)v4.w - va), cf[3]);
                        }
#pragma unroll
                        for (int q = 0; q < VEC; ++q) v.v[q] = (IT)((U)v.v[q] + (U)(int)cf[q]);
#pragma unroll
                        for (int r = 0; r < CL; ++r)
                            st_async16(A_at[r] + (uint32_t)((p * npad + c4 * VEC) * sizeof(IT)), v,
                                       bar_at[r] + p * 8);
                    }
                }
            }

            // the next location's facility, unchanged unless this update's swap moves it
            const int a_pref = s_phi[inext];
            bool timeout = false;
            if constexpr (CL == 1) {
                G.sync();
            } else {
                timeout = !mbar_wait_bounded(smem_u32(&s_bar[p]), (phase >> p) & 1u, kWaitLimitNs);
                phase ^= 1u << p;
            }
            const int b0 = tid * K;
            IT d[4];
            double x[4];
            IT lmax = 0;                                     // max starts at 0 (:208)
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                d[k] = 0;
                x[k] = 0.0;
                if (k < K && b0 + k < ncand) {
                    const int b = b0 + k;
                    d[k] = (CL == 1) ? s_A[p * npad + b] : (IT)((U)s_A[p * npad + b] + (U)s_B[p * npad + b]);
                    lmax = d[k] > lmax ? d[k] : lmax;
                }
            }
            lmax = warp_max(lmax);
            if (lane == 0) s_red[warp] = lmax;
            if (G.sync_or(timeout)) {
                if (tid == 0) atomicOr(s.error, kErrTimeout);
                failed = true;
                break;
            }
            if (tid == 0) s_misc[0] = 0x7fffffff;
            // the weights do not depend on the maximum: formed while it is read
            const IT M = block_max(s_red, nwarps, lane);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (k < K && b0 + k < ncand) {
                    x[k] = exp2(__dmul_rn(beta, (double)d[k]));
                    if (inact && b0 + k == act) x[k] = __dmul_rn(x[k], (double)(n - act));   // :261-264
                }
            }
            const long long cut = cutoff_trunc(__dsub_rn((double)M, cut_span));   // :234-235
            double pre[4];
            double local = 0.0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const bool lumped = inact && b0 + k == act;      // never cut off (:256)
                if (k < K && ((long long)d[k] > cut || lumped) && b0 + k < ncand) local = __dadd_rn(local, x[k]);
                pre[k] = local;
            }
            double incl = local;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl = __dadd_rn(incl, y);
            }
            double excl = __shfl_up_sync(0xffffffffu, incl, 1);
            if (lane == 0) excl = 0.0;
            if (lane == 31) s_wsum[warp] = incl;
            G.sync();
            double base, total;
            weight_totals(s_wsum, nwarps, warp, base, total);
            const double target = __dmul_rn(s_r[i], total);     // :247
            const double X = __dadd_rn(base, excl);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (k < K && b0 + k < npick) {               // the lumped candidate is not scanned
                    if (__dadd_rn(X, pre[k]) >= target) {   // :251
                        // the candidate with its partner j = phiinv(b), read before anyone swaps
                        atomicMin(&s_misc[0], ((b0 + k) << 9) | s_inv[b0 + k]);
                        break;
                    }
                }
            }
            G.sync();
            const int key = s_misc[0];
            const int bs = key >> 9;
            if (bs >= n && inact) {
                // lumped move between two inactive facilities: energy and forces unchanged
                // (CPU_PIM_tai256c.cpp:323-336)
                if (tid == 0) {
                    const int b = lumped_facility((uint32_t)i, sweep, (uint32_t)l, (uint32_t)g, k0, k1, act,
                                                  (uint32_t)(n - act));
                    const int j = s_inv[b];
                    s_phi[i] = b;
                    s_inv[b] = i;
                    s_phi[j] = a;
                    s_inv[a] = j;
                    if (b != a) ++accepts;                   // tid 0's count is the one stored
                }
                G.sync();
                a_nx = -1;                                   // only thread 0 knows the partner
                if (one_row && tid < rows) bj = s_phi[row0 + tid];
                continue;
            }
            if (bs >= n || bs == a) {                        // no move / self move (:252)
                a_nx = a_pref;
                continue;
            }

            // ---- accepted swap: every row and bit row it needs is already in shared memory
            const int j = key & 511;
            a_nx = inext == j ? a : (inext == i ? bs : a_pref);
            if (one_row && tid < rows) {
                if (row0 + tid == i) bj = bs;
                else if (row0 + tid == j) bj = a;
            }
            const IT dEsel = (CL == 1) ? s_A[p * npad + bs] : (IT)((U)s_A[p * npad + bs] + (U)s_B[p * npad + bs]);
            if (tid == 0) {                                  // :257-261
                s_phi[i] = bs;
                s_inv[bs] = i;
                s_phi[j] = a;
                s_inv[a] = j;
            }
            E -= (int64_t)dEsel;                             // :256
            ++accepts;
            if (E < bestE) {                                 // :271-272
                bestE = E;
                if (tid == 0) s_misc[1] = upd;
            }
            const int16_t *Dj = s_Ds + (size_t)j * rpc;
            if (lazy) {   // log the swap; rewrite the rows once kBinLog swaps are pending
                for (int k = tid; k < rpc; k += BT)
                    s_LU[m * rpc + k] = k < rows ? (float)(2 * ((int)Dj[k] - (int)Di[k])) : 0.0f;
                for (int c = tid; c < npad; c += BT)
                    s_V8[(size_t)m * npad + c] = (int8_t)(c < n ? fbit(bs, c) - fbit(a, c) : 0);
                ++m;
                if (m == kBinLog) {
                    G.sync();
                    flush();
                    m = 0;
                    if (failed) break;                       // the rewrite's MMA did not complete
                }
                G.sync();                                    // log, rows and phi visible
                if (s_misc[1] == upd) {
                    for (int q = tid; q < n; q += BT) s_bphi[q] = s_phi[q];
                }
                continue;
            }
            // I[k][c] += 2 (D[j][k] - D[i][k]) (F[bs][c] - F[a][c]).  With clique flows only
            // columns a and bs change when both facilities are active, and only the active
            // columns when one is (CPU_PIM_tai256c.cpp:286-302): the other differences are 0.
            int nv = nvec;
            if (act > 0) {
                if (a < act && bs < act) {
                    for (int k = tid; k < rows; k += BT) {
                        const U u1 = 2u * ((U)(IT)Dj[k] - (U)(IT)Di[k]);
                        IT *Ik = sI + (size_t)k * lds;
                        Ik[a] = (IT)((U)Ik[a] + u1);         // F[bs][a] - F[a][a] = 1
                        Ik[bs] = (IT)((U)Ik[bs] - u1);       // F[bs][bs] - F[a][bs] = -1
                    }
                    nv = 0;
                } else {
                    nv = min(nvec, (act + VEC - 1) / VEC);
                }
            }
            for (int cv = tid % nvec, k0r = tid / nvec, kstep = max(1, BT / nvec);
                 cv < nv; cv += (BT >= nvec ? nvec : BT)) {
                if (BT >= nvec && k0r >= kstep) break;
                const int c0 = cv * VEC;
                const unsigned fb = (s_Fb[bs * nw + (c0 >> 5)] >> (c0 & 31)) & 15u;
                const unsigned fa = (s_Fb[a * nw + (c0 >> 5)] >> (c0 & 31)) & 15u;
                U v1[VEC];
#pragma unroll
                for (int q = 0; q < VEC; ++q) v1[q] = (U)((fb >> q) & 1u) - (U)((fa >> q) & 1u);
                const int kfirst = (BT >= nvec) ? k0r : 0;
                const int kinc = (BT >= nvec) ? kstep : 1;
                constexpr int RB = 8;
                int k = kfirst;
                for (; k + (RB - 1) * kinc < rows; k += RB * kinc) {
                    Vec<IT> xv[RB];
#pragma unroll
                    for (int m = 0; m < RB; ++m)
                        xv[m] = *reinterpret_cast<const Vec<IT> *>(sI + (size_t)(k + m * kinc) * lds + c0);
#pragma unroll
                    for (int m = 0; m < RB; ++m) {
                        const int kk = k + m * kinc;
                        const U u1 = 2u * ((U)(IT)Dj[kk] - (U)(IT)Di[kk]);
#pragma unroll
                        for (int q = 0; q < VEC; ++q) xv[m].v[q] = (IT)((U)xv[m].v[q] + u1 * v1[q]);
                    }
#pragma unroll
                    for (int m = 0; m < RB; ++m)
                        *reinterpret_cast<Vec<IT> *>(sI + (size_t)(k + m * kinc) * lds + c0) = xv[m];
                }
                for (; k < rows; k += kinc) {
                    Vec<IT> *dst = reinterpret_cast<Vec<IT> *>(sI + (size_t)k * lds + c0);
                    Vec<IT> xv = *dst;
                    const U u1 = 2u * ((U)(IT)Dj[k] - (U)(IT)Di[k]);
#pragma unroll
                    for (int q = 0; q < VEC; ++q) xv.v[q] = (IT)((U)xv.v[q] + u1 * v1[q]);
                    *dst = xv;
                }
            }
            G.sync();                                        // new rows and phi visible
            if (s_misc[1] == upd) {
                for (int q = tid; q < n; q += BT) s_bphi[q] = s_phi[q];
            }
        }
    }

    if (m > 0 && !tc_dead) {   // the swaps still pending (m is the same in every thread)
        G.sync();
        flush();
        m = 0;
        G.sync();
    }
    cluster_sync<CL>(G);
    if (tcr) {   // every tensor-memory read has completed (tcgen05.wait::ld, fence, barrier)
        if (warp == 0) {
            // after a wait that gave up, one more bounded wait for the MMA still in flight
            if (tc_dead) mbar_wait_bounded(tc_bar, tc_phase ^ 1u, kWaitLimitNs);
            tc_fence_after();
            tmem_dealloc(tmem, tcols);
        }
        if (tid == 0) mbar_inval(tc_bar);
    }
    if constexpr (CL > 1) {
        if (tid == 0) {
            mbar_inval(smem_u32(&s_bar[0]));
            mbar_inval(smem_u32(&s_bar[1]));
        }
    }
    if (failed) return false;
    {
        IT *gI = reinterpret_cast<IT *>(s.I) + ((size_t)rep * n + row0) * s.ldg;
        const int nvg = s.ldg / VEC;
        for (int idx = tid; idx < rows * nvg; idx += BT) {
            const int k = idx / nvg, v = idx - k * nvg;
            *reinterpret_cast<Vec<IT> *>(gI + (size_t)k * s.ldg + v * VEC) =
                *reinterpret_cast<const Vec<IT> *>(sI + (size_t)k * lds + v * VEC);
        }
    }
    if (rank == 0) {
        int32_t *gphi = s.phi + (size_t)rep * n;
        for (int q = tid; q < n; q += BT) gphi[q] = s_phi[q];
        if (s_misc[1] >= 0) {
            int32_t *gb = s.best_phi + (size_t)rep * n;
            for (int q = tid; q < n; q += BT) gb[q] = s_bphi[q];
        }
        if (tid == 0) {
            s.E[rep] = E;
            s.bestE[rep] = bestE;
            s.accepts[rep] = __ldcg(s.accepts + rep) + accepts;
        }
    }
    __threadfence();
    return true;
}

// ------------------------------------------------------------------ the pipelined binary-flow epoch

// replica_epoch_bin with the deltas of update u + 1 computed while update u picks.  The CTA's
// 256 threads are two groups: the pick group (threads 0-127, named barrier 1) forms the weights,
// the prefix sums and the pick of update u; meanwhile the delta group (threads 128-255, named
// barrier 2) computes the deltas of update u + 1 against the state before update u's swap
// (Bpre / Apre).  Once the pick is known (CTA barrier 1), the delta group applies the swap,
// adds the new log entry's term to every delta, recomputes the two rows whose facilities moved
// (every delta when the next location is the swap partner, whose facility changed), and pushes
// them (CTA barrier 2); the pick group writes the entry's column factors meanwhile.  Same integers,
// weights, sums and picks as replica_epoch_bin; two CTA barriers per update instead of four.
// The uniform r of update u + 1 is drawn by the delta group during update u.
struct PipeLayout {
    size_t I, phi, inv, bphi, Dd, A, B, Bpre, Apre, Ds, Fb, LU, V8, red, wsum, r, misc, bar, total;
    __host__ __device__ PipeLayout(int n, int rpc, int lds) {
        const size_t npad = (size_t)((n + 3) & ~3), rp = (size_t)rpc, nw = (size_t)((n + 31) / 32);
        size_t o = 0;
        I = o;     o = align16(o + rp * lds * 4);
        phi = o;   o = align16(o + npad * 4);
        inv = o;   o = align16(o + npad * 4);
        bphi = o;  o = align16(o + npad * 4);
        Dd = o;    o = align16(o + npad * 4);
        A = o;     o = align16(o + 2 * npad * 4);           // [2][npad] by update parity
        B = o;     o = align16(o + 2 * npad * 4);
        Bpre = o;  o = align16(o + rp * 4);                 // next update's B of this CTA's rows
        Apre = o;  o = align16(o + npad * 4);               // next update's A (owner of its row)
        Ds = o;    o = align16(o + (size_t)n * rp * 2);
        Fb = o;    o = align16(o + (size_t)n * nw * 4);
        LU = o;    o = align16(o + (size_t)kBinLog * rp * 4);
        V8 = o;    o = align16(o + (size_t)kBinLog * npad);
        red = o;   o = align16(o + kMaxWarps * 8);
        wsum = o;  o = align16(o + kMaxWarps * sizeof(double));
        r = o;     o = align16(o + 2 * sizeof(double));      // r of the current / next update
        misc = o;  o = align16(o + 4 * sizeof(int));
        bar = o;   o = align16(o + 2 * sizeof(unsigned long long));
        total = o;
    }
};

size_t epoch_smem_bytes_pipe(int n, int rpc, int lds) { return PipeLayout(n, rpc, lds).total; }

constexpr int kPipeGroup = 128;   // threads of each group of the pipelined epoch

// The rewrite of the CTA's force rows with the m pending log entries, by every thread of the
// CTA: I[k][c] += sum_p LU[p][k] V8[p][c], 8 rows x 4 columns of binary32 sums per thread (exact:
// every partial sum stays below 2^24, as in replica_epoch_bin).
__device__ void pipe_flush(int32_t *sI, const float *s_LU, const int8_t *s_V8, int rows, int rpc, int lds,
                           int npad, int m) {
    constexpr int VEC = 4, RT = 8;
    const int tid = (int)threadIdx.x, BT = (int)blockDim.x;
    const int nvec = npad / VEC;
    const int ngroups = max(1, BT / nvec);                   // row-block groups in flight
    for (int cv = tid % nvec, grp = tid / nvec; cv < nvec; cv += (BT >= nvec ? nvec : BT)) {
        if (BT >= nvec && grp >= ngroups) break;
        const int c0 = cv * VEC;
        const int gfirst = (BT >= nvec) ? grp : 0, ginc = (BT >= nvec) ? ngroups : 1;
        for (int kb = gfirst * RT; kb < rows; kb += ginc * RT) {
            float acc[RT][VEC];
#pragma unroll
            for (int r = 0; r < RT; ++r)
#pragma unroll
                for (int q = 0; q < VEC; ++q) acc[r][q] = 0.0f;
            for (int p = 0; p < m; ++p) {
                const char4 v4 = *reinterpret_cast<const char4 *>(s_V8 + (size_t)p * npad + c0);
                const float v[VEC] = {(float)v4.x, (float)v4.y, (float)v4.z, (float)v4.w};
                // LU rows are rpc long (a multiple of 4): rows past `rows` hold zeros
                const float4 l0 = *reinterpret_cast<const float4 *>(s_LU + (size_t)p * rpc + kb);
                const float4 l1 = (kb + 4 < rpc) ? *reinterpret_cast<const float4 *>(s_LU + (size_t)p * rpc + kb + 4)
                                                 : make_float4(0.f, 0.f, 0.f, 0.f);
                const float u[RT] = {l0.x, l0.y, l0.z, l0.w, l1.x, l1.y, l1.z, l1.w};
#pragma unroll
                for (int r = 0; r < RT; ++r)
#pragma unroll
                    for (int q = 0; q < VEC; ++q) acc[r][q] = fmaf(u[r], v[q], acc[r][q]);
            }
#pragma unroll
            for (int r = 0; r < RT; ++r) {
                if (kb + r < rows) {
                    Vec<int32_t> *dst = reinterpret_cast<Vec<int32_t> *>(sI + (size_t)(kb + r) * lds + c0);
                    Vec<int32_t> xv = *dst;
#pragma unroll
                    for (int q = 0; q < VEC; ++q) xv.v[q] = (int32_t)((uint32_t)xv.v[q] + (uint32_t)(int)acc[r][q]);
                    *dst = xv;
                }
            }
        }
    }
}

// One epoch of replica rep (blockDim.x == 2 * kPipeGroup; symmetric 0/1 flows, int16
// distances, int32 forces, no clique moves).  Returns false when a bounded wait gave up.
template <int CL>
__device__ bool replica_epoch_pipe(const SolveDev &s, int rep, int rank, int e, unsigned char *smem) {
    using IT = int32_t;
    using U = uint32_t;
    constexpr int VEC = 4;
    const int n = s.n;
    const int tid = (int)threadIdx.x, lane = tid & 31;
    const bool pick_group = tid < kPipeGroup;
    const int gt = pick_group ? tid : tid - kPipeGroup;         // thread within its group
    const Grp P{gt, kPipeGroup, lane, gt >> 5, kPipeGroup / 32, 1};
    const Grp Dg{gt, kPipeGroup, lane, gt >> 5, kPipeGroup / 32, 2};
    const int g = rep / s.R, l = rep - g * s.R;
    const int rpc = s.rpc, lds = s.lds;
    const int row0 = rank * rpc;
    const int rows = max(0, min(rpc, n - row0));
    const int npad = (n + 3) & ~3, nvec = npad / VEC;
    const int nw = (n + 31) / 32;
    const PipeLayout L(n, rpc, lds);
    IT *sI = reinterpret_cast<IT *>(smem + L.I);
    int32_t *s_phi = reinterpret_cast<int32_t *>(smem + L.phi);
    int32_t *s_inv = reinterpret_cast<int32_t *>(smem + L.inv);
    int32_t *s_bphi = reinterpret_cast<int32_t *>(smem + L.bphi);
    int32_t *s_Dd = reinterpret_cast<int32_t *>(smem + L.Dd);
    IT *s_A = reinterpret_cast<IT *>(smem + L.A);
    IT *s_B = reinterpret_cast<IT *>(smem + L.B);
    IT *s_Bpre = reinterpret_cast<IT *>(smem + L.Bpre);
    IT *s_Apre = reinterpret_cast<IT *>(smem + L.Apre);
    int16_t *s_Ds = reinterpret_cast<int16_t *>(smem + L.Ds);
    uint32_t *s_Fb = reinterpret_cast<uint32_t *>(smem + L.Fb);
    float *s_LU = reinterpret_cast<float *>(smem + L.LU);
    int8_t *s_V8 = reinterpret_cast<int8_t *>(smem + L.V8);
    IT *s_red = reinterpret_cast<IT *>(smem + L.red);
    double *s_wsum = reinterpret_cast<double *>(smem + L.wsum);
    double *s_r = reinterpret_cast<double *>(smem + L.r);
    int *s_misc = reinterpret_cast<int *>(smem + L.misc);   // [0] pick key, [1] improved at, [2] failed
    unsigned long long *s_bar = reinterpret_cast<unsigned long long *>(smem + L.bar);
    auto fbit = [&](int a, int b) -> int { return (int)((s_Fb[a * nw + (b >> 5)] >> (b & 31)) & 1u); };

    // ---- load the replica and the instance (every thread)
    {
        const IT *gI = reinterpret_cast<const IT *>(s.I) + ((size_t)rep * n + row0) * s.ldg;
        const int nvg = s.ldg / VEC;
        for (int idx = tid; idx < rows * nvg; idx += blockDim.x) {
            const int k = idx / nvg, v = idx - k * nvg;
            const int4 w = __ldcg(reinterpret_cast<const int4 *>(gI + (size_t)k * s.ldg + v * VEC));
            *reinterpret_cast<int4 *>(sI + (size_t)k * lds + v * VEC) = w;
        }
        const int32_t *gphi = s.phi + (size_t)rep * n;
        for (int q = tid; q < npad; q += blockDim.x) {
            int p = q < n ? __ldcg(gphi + q) : 0;
            if ((unsigned)p >= (unsigned)n) {
                atomicOr(s.error, kErrBadPerm);
                p = 0;
            }
            s_phi[q] = p;
            s_bphi[q] = p;
            s_inv[q] = 0;
            s_Dd[q] = q < n ? __ldcg(s.Ddiag + q) : 0;
        }
        load_bin_instance(s, rank, tid, (int)blockDim.x, lane, tid >> 5, (int)(blockDim.x >> 5), s_Ds, s_Fb);
        if (tid == 0) {
            s_misc[0] = 0x7fffffff;
            s_misc[1] = -1;
            s_misc[2] = 0;
            if constexpr (CL > 1) {
                mbar_init(smem_u32(&s_bar[0]), 1);
                mbar_init(smem_u32(&s_bar[1]), 1);
                mbar_fence_init();
            }
        }
        __syncthreads();
    }
    for (int q = tid; q < n; q += blockDim.x) s_inv[s_phi[q]] = q;
    cluster_sync<CL>(Grp{tid, (int)blockDim.x, lane, tid >> 5, (int)(blockDim.x >> 5), 0});

    uint32_t A_at[CL], B_at[CL], bar_at[CL];
    if constexpr (CL > 1) {
#pragma unroll
        for (int r = 0; r < CL; ++r) {
            A_at[r] = cluster_addr(smem_u32(s_A), r);
            B_at[r] = cluster_addr(smem_u32(s_B), r);
            bar_at[r] = cluster_addr(smem_u32(s_bar), r);
        }
    }
    const uint32_t tx_bytes = (uint32_t)((npad + n) * sizeof(IT));
    uint32_t phase = 0;
    const double beta = __ldcg(s.beta + rep);
    const double cut_span = 20.0 / beta;                    // CPU_PIM.cpp:234
    int64_t E = __ldcg((const long long *)s.E + rep), bestE = __ldcg((const long long *)s.bestE + rep);
    unsigned long long accepts = 0;
    const uint32_t k0 = (uint32_t)s.seed, k1 = (uint32_t)(s.seed >> 32);
    const int K = (n + kPipeGroup - 1) / kPipeGroup;         // weights per pick thread (<= 4)
    const int U_total = s.spe * n;                           // updates of this epoch
    int m = 0;                                               // pending swaps (same in every thread)

    // The uniform r of update u (:212): the caller's or the Philox stream's.
    auto draw_r = [&](int u) -> double {
        const int i = u % n;
        const uint32_t sweep = (uint32_t)(e * s.spe + u / n);
        if (s.replay_r) return __ldcg(s.replay_r + (size_t)sweep * n + i);
        uint32_t w0, w1;
        philox_2words((uint32_t)i, sweep, (uint32_t)l, (uint32_t)g, k0, k1, w0, w1);
        return canonical53(w0, w1);
    };
    // The swap log's correction of a B-half entry (row jj, candidate b, facility a1 at the
    // updating location) and of an A-half entry (row il of that location, column c), over the
    // m pending entries (binary32 sums, exact as in replica_epoch_bin).
    auto corr_B = [&](int jj, int a1, int b) -> int {
        float cf = 0.0f;
#pragma unroll 4
        for (int q = 0; q < m; ++q) {
            const int8_t *v8 = s_V8 + (size_t)q * npad;
            cf = fmaf(s_LU[q * rpc + jj], (float)((int)v8[a1] - (int)v8[b]), cf);
        }
        return (int)cf;
    };
    // B-half of row jj for the update of location i1 (facility a1), candidate b = its facility:
    // I[j][a1] - I[j][b] - dd ff with the log's corrections.
    auto row_B = [&](int i1, int a1, int jj, int b) -> U {
        const int j = row0 + jj;
        const IT *Ij = sI + (size_t)jj * lds;
        const U dd = (U)s_Dd[i1] + (U)s_Dd[j] - 2u * (U)(IT)s_Ds[(size_t)i1 * rpc + jj];
        const U ff = (U)fbit(a1, a1) + (U)fbit(b, b) - 2u * (U)fbit(a1, b);
        return (U)Ij[a1] - (U)Ij[b] - dd * ff + (U)corr_B(jj, a1, b);
    };
    // A-half of the update of location i1 (facility a1), columns 4 c4 .. 4 c4 + 3, by the owner
    // of row i1: I[i1][c] - I[i1][a1] with the log's corrections.
    auto chunk_A = [&](int i1, int a1, int c4) -> Vec<IT> {
        const int il = i1 - row0;
        const IT *Ii = sI + (size_t)il * lds;
        const IT Iia = Ii[a1];
        Vec<IT> v = *reinterpret_cast<const Vec<IT> *>(Ii + c4 * VEC);
        const int c0 = c4 * VEC;
        float cf[VEC] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll 4
        for (int q = 0; q < m; ++q) {
            const int8_t *v8 = s_V8 + (size_t)q * npad;
            const char4 v4 = *reinterpret_cast<const char4 *>(v8 + c0);
            const int va = (int)v8[a1];
            const float lu = s_LU[q * rpc + il];
            cf[0] = fmaf(lu, (float)((int)v4.x - va), cf[0]);
            cf[1] = fmaf(lu, (float)((int)v4.y - va), cf[1]);
            cf[2] = fmaf(lu, (float)((int)v4.z - va), cf[2]);
            cf[3] = fmaf(lu, (float)((int)v4.w - va), cf[3]);
        }
#pragma unroll
        for (int q = 0; q < VEC; ++q) v.v[q] = (IT)((U)v.v[q] - (U)Iia + (U)(int)cf[q]);
        return v;
    };
    // Update u1's halves into the receive buffers of parity p1 of every CTA of the cluster.
    auto push_B = [&](int p1, int b, IT v) {
        if constexpr (CL == 1) {
            s_B[p1 * npad + b] = v;
        } else {
#pragma unroll
            for (int r = 0; r < CL; ++r)
                st_async(B_at[r] + (uint32_t)((p1 * npad + b) * sizeof(IT)), v, bar_at[r] + p1 * 8);
        }
    };
    auto push_A = [&](int p1, int c4, const Vec<IT> &v) {
        if constexpr (CL == 1) {
            *reinterpret_cast<Vec<IT> *>(s_A + p1 * npad + c4 * VEC) = v;
        } else {
#pragma unroll
            for (int r = 0; r < CL; ++r)
                st_async16(A_at[r] + (uint32_t)((p1 * npad + c4 * VEC) * sizeof(IT)), v, bar_at[r] + p1 * 8);
        }
    };

    // ---- update 0's deltas (no swap before it) and r
    if (!pick_group) {
        const int a0 = s_phi[0];
        for (int jj = gt; jj < rows; jj += kPipeGroup) push_B(0, s_phi[row0 + jj], (IT)row_B(0, a0, jj, s_phi[row0 + jj]));
        if (0 / rpc == rank)
            for (int c4 = gt; c4 < nvec; c4 += kPipeGroup) push_A(0, c4, chunk_A(0, a0, c4));
        if (gt == kPipeGroup - 1) s_r[0] = draw_r(0);
    } else if (CL > 1 && gt == 0) {
        mbar_arrive_expect_tx(smem_u32(&s_bar[0]), tx_bytes);
    }
    __syncthreads();

    bool failed = false;
    for (int u = 0; u < U_total; ++u) {
        const int i = u % n;
        const int p = u & 1;
        const int a = s_phi[i];
        const bool has_next = u + 1 < U_total;
        const int i1 = has_next ? (u + 1) % n : 0;
        const int a1 = has_next ? s_phi[i1] : 0;            // before update u's swap
        // ---- phase A: the pick of update u | the deltas of update u + 1
        if (pick_group) {
            bool timeout = false;
            if constexpr (CL > 1) {
                timeout = !mbar_wait_bounded(smem_u32(&s_bar[p]), (phase >> p) & 1u, kWaitLimitNs);
                phase ^= 1u << p;
            }
            const int b0 = gt * K;
            IT d[4];
            double x[4];
            IT lmax = 0;                                     // max starts at 0 (:208)
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                d[k] = 0;
                x[k] = 0.0;
                if (k < K && b0 + k < n) {
                    const int b = b0 + k;
                    d[k] = (IT)((U)s_A[p * npad + b] + (U)s_B[p * npad + b]);
                    x[k] = exp2(__dmul_rn(beta, (double)d[k]));
                    lmax = d[k] > lmax ? d[k] : lmax;
                }
            }
            lmax = warp_max(lmax);
            if (lane == 0) s_red[P.warp] = lmax;
            if (P.sync_or(timeout)) {
                if (gt == 0) {
                    atomicOr(s.error, kErrTimeout);
                    s_misc[2] = 1;
                }
            } else {
                if (gt == 0) s_misc[0] = 0x7fffffff;
                IT M = s_red[0];
                for (int w = 1; w < P.nwarps; ++w) M = s_red[w] > M ? s_red[w] : M;
                const long long cut = cutoff_trunc(__dsub_rn((double)M, cut_span));   // :234-235
                double pre[4];
                double local = 0.0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (k < K && (long long)d[k] > cut && b0 + k < n) local = __dadd_rn(local, x[k]);
                    pre[k] = local;
                }
                double incl = local;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const double y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl = __dadd_rn(incl, y);
                }
                double excl = __shfl_up_sync(0xffffffffu, incl, 1);
                if (lane == 0) excl = 0.0;
                if (lane == 31) s_wsum[P.warp] = incl;
                P.sync();
                double base = 0.0, total = 0.0;
                for (int w = 0; w < P.nwarps; ++w) {
                    if (w == P.warp) base = total;
                    total = __dadd_rn(total, s_wsum[w]);
                }
                const double target = __dmul_rn(s_r[p], total);      // :247
                const double X = __dadd_rn(base, excl);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (k < K && b0 + k < n) {
                        if (__dadd_rn(X, pre[k]) >= target) {    // :251
                            atomicMin(&s_misc[0], ((b0 + k) << 9) | s_inv[b0 + k]);
                            break;
                        }
                    }
                }
            }
        } else if (has_next) {
            for (int jj = gt; jj < rows; jj += kPipeGroup) s_Bpre[jj] = (IT)row_B(i1, a1, jj, s_phi[row0 + jj]);
            if (i1 / rpc == rank)
                for (int c4 = gt; c4 < nvec; c4 += kPipeGroup)
                    *reinterpret_cast<Vec<IT> *>(s_Apre + c4 * VEC) = chunk_A(i1, a1, c4);
            if (gt == kPipeGroup - 1) s_r[p ^ 1] = draw_r(u + 1);
        }
        __syncthreads();                                     // 1: the pick is known
        if (s_misc[2]) {
            failed = true;
            break;
        }
        const int key = s_misc[0];
        const int bs = key >> 9, js = key & 511;
        const bool accepted = bs < n && bs != a;             // no move / self move (:252)
        if (accepted) {
            E -= (int64_t)(IT)((U)s_A[p * npad + bs] + (U)s_B[p * npad + bs]);   // :256
            ++accepts;
            if (E < bestE) {                                 // :271-272
                bestE = E;
                if (tid == 0) s_misc[1] = u;
            }
        }
        // ---- phase B: the log entry of the swap | update u + 1's deltas completed and pushed
        if (pick_group) {
            if (CL > 1 && has_next && gt == 0) mbar_arrive_expect_tx(smem_u32(&s_bar[p ^ 1]), tx_bytes);
            if (accepted)
                for (int c = gt; c < npad; c += kPipeGroup)
                    s_V8[(size_t)m * npad + c] = (int8_t)(c < n ? fbit(bs, c) - fbit(a, c) : 0);
        } else {
            if (accepted) {
                if (gt == 0) {                               // :257-261
                    s_phi[i] = bs;
                    s_inv[bs] = i;
                    s_phi[js] = a;
                    s_inv[a] = js;
                }
                for (int k = gt; k < rpc; k += kPipeGroup)
                    s_LU[m * rpc + k] =
                        k < rows ? (float)(2 * ((int)s_Ds[(size_t)js * rpc + k] - (int)s_Ds[(size_t)i * rpc + k])) : 0.0f;
            }
            if (has_next) {
                const int p1 = p ^ 1;
                // the new entry's row factor 2 (D[k][js] - D[k][i]) and column factor F[bs][c] - F[a][c]
                auto lux = [&](int kk) -> int { return 2 * ((int)s_Ds[(size_t)js * rpc + kk] - (int)s_Ds[(size_t)i * rpc + kk]); };
                auto vx = [&](int c) -> int { return fbit(bs, c) - fbit(a, c); };
                const bool full = accepted && i1 == js;      // location i1 now holds facility a
                const int a1n = full ? a : a1;
                for (int jj = gt; jj < rows; jj += kPipeGroup) {
                    const int j = row0 + jj;
                    const bool moved = accepted && (j == i || j == js);
                    const int b = moved ? (j == i ? bs : a) : s_phi[j];   // rows i / js: being rewritten
                    U v = (full || moved) ? row_B(i1, a1n, jj, b) : (U)s_Bpre[jj];
                    if (accepted) v += (U)(lux(jj) * (vx(a1n) - vx(b)));
                    push_B(p1, b, (IT)v);
                }
                if (i1 / rpc == rank) {
                    const int il = i1 - row0;
                    for (int c4 = gt; c4 < nvec; c4 += kPipeGroup) {
                        Vec<IT> v = full ? chunk_A(i1, a1n, c4) : *reinterpret_cast<const Vec<IT> *>(s_Apre + c4 * VEC);
                        if (accepted) {
                            const int lx = lux(il), va = vx(a1n);
#pragma unroll
                            for (int q = 0; q < VEC; ++q) {
                                const int c = c4 * VEC + q;
                                v.v[q] = (IT)((U)v.v[q] + (U)(lx * ((c < n ? vx(c) : 0) - va)));
                            }
                        }
                        push_A(p1, c4, v);
                    }
                }
            }
        }
        __syncthreads();                                     // 2: swap, log entry and pushes done
        if (accepted) ++m;
        if (s_misc[1] == u)
            for (int q = tid; q < n; q += blockDim.x) s_bphi[q] = s_phi[q];
        if (m == kBinLog) {
            pipe_flush(sI, s_LU, s_V8, rows, rpc, lds, npad, m);
            m = 0;
            __syncthreads();
        }
    }
    if (!failed && m > 0) {   // the swaps still pending (m is the same in every thread)
        pipe_flush(sI, s_LU, s_V8, rows, rpc, lds, npad, m);
        m = 0;
        __syncthreads();
    }
    cluster_sync<CL>(Grp{tid, (int)blockDim.x, lane, tid >> 5, (int)(blockDim.x >> 5), 0});
    if constexpr (CL > 1) {
        if (tid == 0) {
            mbar_inval(smem_u32(&s_bar[0]));
            mbar_inval(smem_u32(&s_bar[1]));
        }
    }
    if (failed) return false;
    {
        IT *gI = reinterpret_cast<IT *>(s.I) + ((size_t)rep * n + row0) * s.ldg;
        const int nvg = s.ldg / VEC;
        for (int idx = tid; idx < rows * nvg; idx += blockDim.x) {
            const int k = idx / nvg, v = idx - k * nvg;
            *reinterpret_cast<Vec<IT> *>(gI + (size_t)k * s.ldg + v * VEC) =
                *reinterpret_cast<const Vec<IT> *>(sI + (size_t)k * lds + v * VEC);
        }
    }
    if (rank == 0) {
        int32_t *gphi = s.phi + (size_t)rep * n;
        for (int q = tid; q < n; q += blockDim.x) gphi[q] = s_phi[q];
        if (s_misc[1] >= 0) {
            int32_t *gb = s.best_phi + (size_t)rep * n;
            for (int q = tid; q < n; q += blockDim.x) gb[q] = s_bphi[q];
        }
        if (tid == 0) {
            s.E[rep] = E;
            s.bestE[rep] = bestE;
            s.accepts[rep] = __ldcg(s.accepts + rep) + accepts;
        }
    }
    __threadfence();
    return true;
}

// The tensor-core force update of the one-shot epoch stages 64 factor columns at a time, as
// fp16 rows of kMmaLd halves (144 bytes: the 8 rows and 4 column pairs one fragment load
// touches fall in 32 different banks).
constexpr int kMmaK = 64;
constexpr int kMmaLd = 72;

// The tcgen05 form stages the same 64 factor columns as fp16 core matrices (below): A holds
// 128 rows (the MMA's M; rows past the CTA's are never read back), B the columns rounded up
// to 16 (the MMA's N); one 8-row (8-column) group of 64 factor columns is 1024 bytes.
constexpr int kTcGroupBytes = kMmaK / 8 * 128;
constexpr int kTcABytes = 128 / 8 * kTcGroupBytes;

// os_mma values of SolveDev (the one-shot force update)
constexpr int kOsCudaCores = 0, kOsMmaSync = 1, kOsTcgen05 = 2;

// Shared-memory layout of the one-shot epoch (replica_epoch_os).
//   I       rpc rows of the force matrix; odd row stride lds, so 32 lanes reading one column
//           of 32 rows hit 32 banks
//   phi, inv, bphi, Dd, Fd   permutation, inverse, best permutation, diagonals of D and F
//   diag    I[j][phi(j)] of every location (each CTA stores its rows' entries into all CTAs)
//   tgt, dlt   [2][npad] every location's proposal (partner, delta), stored by the CTA that
//           owns the location into all CTAs; double-buffered by step
//   own     ballot words of the collision resolution
//   pair    accepted swaps: i, j, phi(i), phi(j) before the step ([4][npad])
//   uni     thresholds of this CTA's locations for the coming step (binary32)
//   T       (xcol) [rpc][(CL-1) rpc]: for each location i of this CTA, column phi(i) of the
//           other CTAs' rows, pushed by those CTAs (coalesced remote stores) after every step
//           that moved something, so the proposals read no remote memory
//   U, V    factors of one chunk of pc accepted swaps: U[p][k] = 2 (D[k][j] - D[k][i]) over
//           this CTA's rows (row stride rpc), V[p][c] = F[c][b] - F[c][a] (row stride 256, zero
//           beyond n); asymmetric instances use U = D[k][j] - D[k][i] and add
//           U2 = D[j][k] - D[i][k], V2 = F[b][c] - F[a][c].  They share T's space: they are
//           live only between a step's proposals and its column exchange.  The tensor-core
//           forms stage their fp16 factors in the same space (mma.sync: rows of kMmaLd
//           halves; tcgen05: core matrices, A then B)
//   part    [CL] every CTA's share of sum_k I[k][phi(k)], then [kMaxWarpsOs] warp sums
//   misc    [kMaxWarpsOs] warp counts of the pair compaction, [8] flags
//   tc      (tcgen05) the mbarrier the MMAs complete on, the tensor-memory address
struct OsLayout {
    size_t I, phi, inv, bphi, Dd, Fd, diag, tgt, dlt, own, pair, uni, T, U, V, U2, V2, part, misc, tc, total;
    int tld;    // row stride of T (elements)
    int tcn;    // tcgen05: the MMA's N (columns rounded up to 16)
    int tcols;  // tcgen05: tensor-memory columns allocated (a power of two, at least 32)
    __host__ __device__ OsLayout(int n, int rpc, int lds, int cluster, int isz, int pc, bool sym, bool xcol,
                                 int mma = kOsCudaCores) {
        const size_t npad = (size_t)((n + 3) & ~3), rp = (size_t)rpc, vld = 256;
        size_t o = 0;
        I = o;    o = align16(o + rp * lds * isz);
        phi = o;  o = align16(o + npad * 4);
        inv = o;  o = align16(o + npad * 4);
        bphi = o; o = align16(o + npad * 4);
        Dd = o;   o = align16(o + npad * 4);
        Fd = o;   o = align16(o + npad * 4);
        diag = o; o = align16(o + npad * isz);
        tgt = o;  o = align16(o + 2 * npad * 4);
        dlt = o;  o = align16(o + 2 * npad * isz);
        own = o;  o = align16(o + npad * 8);
        pair = o; o = align16(o + 4 * npad * 4);
        uni = o;  o = align16(o + npad * 4);
        tld = xcol ? (cluster - 1) * rpc : 0;
        const size_t tbytes = (size_t)rp * tld * isz;
        T = o;
        U = o;
        V = align16(U + (size_t)pc * rp * isz);
        U2 = align16(V + (size_t)pc * vld * isz);
        V2 = align16(U2 + (sym ? 0 : (size_t)pc * rp * isz));
        size_t fend = align16(V2 + (sym ? 0 : (size_t)pc * vld * isz));
        tcn = (n + 15) & ~15;
        tcols = 32;
        while (tcols < tcn) tcols *= 2;
        if (mma == kOsMmaSync) {   // the tensor-core factors (fp16) share the same space
            const size_t mend = align16(U + (size_t)((rpc + 15) & ~15) * kMmaLd * 2 + (size_t)((n + 7) & ~7) * kMmaLd * 2);
            fend = mend > fend ? mend : fend;
        } else if (mma == kOsTcgen05) {
            const size_t mend = align16(U + (size_t)kTcABytes + (size_t)(tcn / 8) * kTcGroupBytes);
            fend = mend > fend ? mend : fend;
        }
        o = align16(fend > o + tbytes ? fend : o + tbytes);
        part = o; o = align16(o + (size_t)(cluster + kMaxWarpsOs) * 8);
        misc = o; o = align16(o + (kMaxWarpsOs + 8) * sizeof(int));
        tc = o;   o = align16(o + (mma == kOsTcgen05 ? 16 : 0));
        total = o;
    }
};

int os_tmem_columns(int n) { return OsLayout(n, 4, 5, 1, 4, 4, true, false, kOsTcgen05).tcols; }

size_t epoch_smem_bytes_os(int n, int rpc, int lds, int cluster, int bits, int chunk, bool sym, bool xcol,
                           int mma) {
    return OsLayout(n, rpc, lds, cluster, bits / 8, chunk, sym, xcol, mma).total;
}

// One m16n8k16 tensor-core product with fp16 inputs and fp32 accumulation: d += a b.
__device__ __forceinline__ void mma_16816(float d[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
        "{%8, %9}, {%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Eight int32 differences hi - lo (times `scale`) as eight fp16 in one 16-byte word (exact for
// integers of at most 2048 in magnitude).
__device__ __forceinline__ uint4 pack_half8(const int4 &h0, const int4 &l0, const int4 &h1, const int4 &l1,
                                            int scale) {
    const __half2 a = __halves2half2(__int2half_rn(scale * (h0.x - l0.x)), __int2half_rn(scale * (h0.y - l0.y)));
    const __half2 b = __halves2half2(__int2half_rn(scale * (h0.z - l0.z)), __int2half_rn(scale * (h0.w - l0.w)));
    const __half2 c = __halves2half2(__int2half_rn(scale * (h1.x - l1.x)), __int2half_rn(scale * (h1.y - l1.y)));
    const __half2 d = __halves2half2(__int2half_rn(scale * (h1.z - l1.z)), __int2half_rn(scale * (h1.w - l1.w)));
    uint4 r;
    r.x = *reinterpret_cast<const uint32_t *>(&a);
    r.y = *reinterpret_cast<const uint32_t *>(&b);
    r.z = *reinterpret_cast<const uint32_t *>(&c);
    r.w = *reinterpret_cast<const uint32_t *>(&d);
    return r;
}

// Loads of this CTA's shared memory by 32-bit shared address.
template <class IT> __device__ __forceinline__ IT lds_it(uint32_t a);
template <> __device__ __forceinline__ int32_t lds_it<int32_t>(uint32_t a) {
    int32_t v;
    asm volatile("ld.shared.b32 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}
template <> __device__ __forceinline__ int64_t lds_it<int64_t>(uint32_t a) {
    long long v;
    asm volatile("ld.shared.b64 %0, [%1];" : "=l"(v) : "r"(a));
    return (int64_t)v;
}

// Loads / stores of another CTA's shared memory (shared::cluster addresses from mapa).
__device__ __forceinline__ int32_t ld_cluster(uint32_t a, int32_t) {
    int32_t v;
    asm volatile("ld.shared::cluster.b32 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ int64_t ld_cluster(uint32_t a, int64_t) {
    long long v;
    asm volatile("ld.shared::cluster.b64 %0, [%1];" : "=l"(v) : "r"(a));
    return (int64_t)v;
}
__device__ __forceinline__ void st_cluster(uint32_t a, int32_t v) {
    asm volatile("st.shared::cluster.b32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ void st_cluster(uint32_t a, int64_t v) {
    asm volatile("st.shared::cluster.b64 [%0], %1;" ::"r"(a), "l"((long long)v) : "memory");
}

// Ballot word of a proposal (i -> partner with delta): the smaller word wins, i.e. the larger
// delta, then the lower i (GPU-CUPIM qap.cu:1184-1198); deltas beyond int32 saturate.
template <class IT> __device__ __forceinline__ unsigned long long oneshot_ballot(IT delta, int i) {
    const long long d = (long long)delta;
    const int32_t d32 = d > 2147483647ll ? 2147483647 : (d < -2147483648ll ? (int32_t)0x80000000 : (int32_t)d);
    const uint32_t biased = ~((uint32_t)d32 ^ 0x80000000u);
    return ((unsigned long long)biased << 32) | (uint32_t)i;
}

// Factors of cn accepted swaps for the one-shot force update, from 16-byte pieces of two rows
// per swap: out[p][4 q + r] = M1[y_p][4 q + r] - M1[x_p][4 q + r] (q < nq), doubled when TWICE
// (the row factors of a symmetric instance, whose two rank-1 terms per swap are equal), and for
// asymmetric instances out2 from M2 likewise.  UNR pieces per thread are loaded before any is
// used.
template <class IT, bool SYM, bool TWICE, int UNR>
__device__ __forceinline__ void stage_factors(int tid, int BT, int cn, int nq, const int32_t *M1,
                                              const int32_t *M2, int ldm, const int32_t *x,
                                              const int32_t *y, IT *out, IT *out2, int ld_out) {
    using U = typename Unsigned<IT>::type;
    const int total = cn * nq;
    for (int base = tid; base < total; base += UNR * BT) {
        int4 hi[UNR], lo[UNR], hi2[UNR], lo2[UNR];
#pragma unroll
        for (int m = 0; m < UNR; ++m) {
            const int idx = base + m * BT;
            if (idx < total) {
                const int p = idx / nq, q = idx - p * nq;
                const size_t ry = (size_t)y[p] * ldm + 4 * q, rx = (size_t)x[p] * ldm + 4 * q;
                hi[m] = __ldg(reinterpret_cast<const int4 *>(M1 + ry));
                lo[m] = __ldg(reinterpret_cast<const int4 *>(M1 + rx));
                if constexpr (!SYM) {
                    hi2[m] = __ldg(reinterpret_cast<const int4 *>(M2 + ry));
                    lo2[m] = __ldg(reinterpret_cast<const int4 *>(M2 + rx));
                }
            }
        }
#pragma unroll
        for (int m = 0; m < UNR; ++m) {
            const int idx = base + m * BT;
            if (idx < total) {
                const int p = idx / nq, q = idx - p * nq;
                IT *o = out + (size_t)p * ld_out + 4 * q;
                const int32_t *h = &hi[m].x, *l = &lo[m].x;
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const U d = (U)(IT)h[r] - (U)(IT)l[r];
                    o[r] = TWICE ? (IT)(2u * d) : (IT)d;
                }
                if constexpr (!SYM) {
                    IT *o2 = out2 + (size_t)p * ld_out + 4 * q;
                    const int32_t *h2 = &hi2[m].x, *l2 = &lo2[m].x;
#pragma unroll
                    for (int r = 0; r < 4; ++r) o2[r] = (IT)((U)(IT)h2[r] - (U)(IT)l2[r]);
                }
            }
        }
    }
}

// One epoch of replica rep under the one-shot parallel update of GPU-CUPIM (qap.cu:1038-1458):
// spe steps, each of which lets every location propose a partner against the same snapshot,
// resolves the collisions, applies the surviving (disjoint) swaps together and recomputes the
// energy from the force matrix.  The replica's force matrix stays resident in shared memory,
// split by rows over the cluster as in the sequential epoch.  Per step:
//   1. proposals: one warp per location i of this CTA; lane t evaluates partners j = t + 32k
//      (the reference's lane layout), reading column phi(i) of the other CTAs' rows through
//      distributed shared memory; binary32 weights 2^(beta (d - max)) by CUDA's exp2f as the
//      reference computes them, or by this library's exp2f_neg (which the oracle restates),
//      the reference's per-lane running sums and 32-lane scan, the threshold pick; the lane
//      that owns location i stores the proposal into every CTA; cluster barrier;
//   2. every CTA resolves all n proposals (shared-memory atomicMin on ballot words, same
//      result everywhere) and compacts the accepted swaps in location order;
//   3. the force update of this CTA's rows, sum over swaps p of U[p][k] V[p][c] (rank-2 per
//      swap), in chunks of pc swaps with RT x 8 register tiles per lane;
//   4. the new diagonal I[k][phi(k)] of this CTA's rows and its share of the energy go to
//      every CTA; cluster barrier; E = -1/2 sum.  A step without swaps skips 3-4.
template <class IT, int CL, bool SYM, bool GP>
__device__ bool replica_epoch_os(const SolveDev &s, int rep, int rank, int e, const Grp &G,
                                 unsigned char *smem) {
    using U = typename Unsigned<IT>::type;
    constexpr int VEC = Vec<IT>::kN;
    constexpr int RT = sizeof(IT) == 4 ? 4 : 2;              // rows of a register tile
    const int n = s.n;
    const int tid = G.tid, BT = G.BT, lane = G.lane, warp = G.warp, nwarps = G.nwarps;
    const int g = rep / s.R, l = rep - g * s.R;
    const int rpc = s.rpc, lds = s.lds, ldm = s.ldm, pc = s.os_chunk;
    const int row0 = rank * rpc;
    const int rows = max(0, min(rpc, n - row0));
    const int npad = (n + 3) & ~3, vld = 256;           // V rows: every lane's 8 columns
    const int K = (n + 31) >> 5;                             // partners per lane (<= 8)
    const bool xcol = CL > 1 && s.os_xcol != 0;
    const bool tc = s.os_mma == kOsTcgen05;
    const bool own_exp2 = s.os_own_exp2 != 0;
    const bool mma = s.os_mma == kOsMmaSync;
    const OsLayout L(n, rpc, lds, CL, (int)sizeof(IT), pc, SYM, xcol, tc ? kOsTcgen05 : (mma ? kOsMmaSync : kOsCudaCores));
    const int tld = L.tld;
    IT *sI = reinterpret_cast<IT *>(smem + L.I);
    int32_t *s_phi = reinterpret_cast<int32_t *>(smem + L.phi);
    int32_t *s_inv = reinterpret_cast<int32_t *>(smem + L.inv);
    int32_t *s_bphi = reinterpret_cast<int32_t *>(smem + L.bphi);
    int32_t *s_Dd = reinterpret_cast<int32_t *>(smem + L.Dd);
    int32_t *s_Fd = reinterpret_cast<int32_t *>(smem + L.Fd);
    float *s_uni = reinterpret_cast<float *>(smem + L.uni);
    IT *s_T = reinterpret_cast<IT *>(smem + L.T);
    IT *s_diag = reinterpret_cast<IT *>(smem + L.diag);
    int32_t *s_tgt = reinterpret_cast<int32_t *>(smem + L.tgt);
    IT *s_dlt = reinterpret_cast<IT *>(smem + L.dlt);
    unsigned long long *s_own = reinterpret_cast<unsigned long long *>(smem + L.own);
    int32_t *s_pi = reinterpret_cast<int32_t *>(smem + L.pair);
    int32_t *s_pj = s_pi + npad, *s_pa = s_pj + npad, *s_pb = s_pa + npad;
    IT *s_U = reinterpret_cast<IT *>(smem + L.U);
    IT *s_V = reinterpret_cast<IT *>(smem + L.V);
    IT *s_U2 = reinterpret_cast<IT *>(smem + L.U2);
    IT *s_V2 = reinterpret_cast<IT *>(smem + L.V2);
    long long *s_part = reinterpret_cast<long long *>(smem + L.part);
    int *s_wcnt = reinterpret_cast<int *>(smem + L.misc);
    int *s_flag = s_wcnt + kMaxWarpsOs;                     // [0] goal-print slot

    // ---- load the replica
    {
        const IT *gI = reinterpret_cast<const IT *>(s.I) + ((size_t)rep * n + row0) * s.ldg;
        const int nvg = s.ldg / VEC;
        for (int idx = tid; idx < rows * nvg; idx += BT) {
            const int k = idx / nvg, v = idx - k * nvg;
            const int4 w4 = __ldcg(reinterpret_cast<const int4 *>(gI + (size_t)k * s.ldg + v * VEC));
            Vec<IT> w;
            memcpy(&w, &w4, 16);
#pragma unroll
            for (int q = 0; q < VEC; ++q) sI[(size_t)k * lds + v * VEC + q] = w.v[q];
        }
        const int32_t *gphi = s.phi + (size_t)rep * n;
        for (int q = tid; q < npad; q += BT) {
            int p = q < n ? __ldcg(gphi + q) : 0;
            if ((unsigned)p >= (unsigned)n) {
                atomicOr(s.error, kErrBadPerm);
                p = 0;
            }
            s_phi[q] = p;
            s_bphi[q] = p;
            s_Dd[q] = q < n ? __ldcg(s.Ddiag + q) : 0;
            s_Fd[q] = q < n ? __ldcg(s.Fdiag + q) : 0;
        }
    }
    // tcgen05: the step's force-update sums live in L.tcols tensor-memory columns (warp 0
    // allocates them; the CTA is alone on its SM, so the allocation does not wait), and the
    // MMAs complete on one mbarrier
    const uint32_t tc_bar = smem_u32(smem + L.tc);
    uint32_t tmem = 0, tc_phase = 0;
    bool tc_dead = false;                                    // a wait for the MMAs gave up
    if (tc) {
        if (warp == 0) tmem_alloc(smem_u32(smem + L.tc + 8), (uint32_t)L.tcols);
        if (tid == 0) {
            mbar_init(tc_bar, 1);
            mbar_fence_init();
        }
        tc_fence_before();
    }
    G.sync();
    if (tc) {
        tc_fence_after();
        tmem = *reinterpret_cast<volatile uint32_t *>(smem + L.tc + 8);
    }
    for (int q = tid; q < n; q += BT) s_inv[s_phi[q]] = q;

    // shared::cluster addresses of every CTA's rows and cluster-wide arrays
    uint32_t I_at[CL], diag_at[CL], tgt_at[CL], dlt_at[CL], part_at[CL], T_at[CL];
#pragma unroll
    for (int r = 0; r < CL; ++r) {
        I_at[r] = CL > 1 ? cluster_addr(smem_u32(sI), r) : smem_u32(sI);
        T_at[r] = CL > 1 ? cluster_addr(smem_u32(s_T), r) : smem_u32(s_T);
        diag_at[r] = CL > 1 ? cluster_addr(smem_u32(s_diag), r) : smem_u32(s_diag);
        tgt_at[r] = CL > 1 ? cluster_addr(smem_u32(s_tgt), r) : smem_u32(s_tgt);
        dlt_at[r] = CL > 1 ? cluster_addr(smem_u32(s_dlt), r) : smem_u32(s_dlt);
        part_at[r] = CL > 1 ? cluster_addr(smem_u32(s_part), r) : smem_u32(s_part);
    }
    const uint32_t k0 = (uint32_t)s.seed, k1 = (uint32_t)(s.seed >> 32);
    // thresholds of this CTA's locations for step `step` (one Philox block each)
    auto draw_thresholds = [&](uint32_t step) {
        for (int q = tid; q < rows; q += BT) {
            uint32_t w0, w1;
            philox_2words((uint32_t)(row0 + q), step, (uint32_t)l, (uint32_t)g, k0, k1, w0, w1);
            s_uni[q] = oneshot_uniform(w0);
        }
    };
    // every other CTA q gets T_q[i - q.row0][slot of j] = I[j][phi(i)] for this CTA's rows j
    // and q's locations i: one warp per location, 32 consecutive rows per store (128 bytes)
    auto send_columns = [&]() {
#pragma unroll
        for (int q = 0; q < CL; ++q) {
            if (q == rank) continue;
            const int qrow0 = q * rpc, qrows = max(0, min(rpc, n - qrow0));
            const int jr0 = row0 < qrow0 ? row0 : row0 - rpc;
            for (int il = warp; il < qrows; il += nwarps) {
                const int a = s_phi[qrow0 + il];
                for (int jl = lane; jl < rows; jl += 32)
                    st_cluster(T_at[q] + (uint32_t)(((size_t)il * tld + jr0 + jl) * sizeof(IT)),
                               sI[(size_t)jl * lds + a]);
            }
        }
    };
    draw_thresholds((uint32_t)(e * s.spe));
    cluster_sync<CL>(G);   // every CTA of the cluster is running before any remote access
    // the diagonal of this CTA's rows into every CTA
    for (int kk = tid; kk < rows; kk += BT) {
        const int k = row0 + kk;
        const IT dv = sI[(size_t)kk * lds + s_phi[k]];
        if constexpr (CL == 1) s_diag[k] = dv;
        else
#pragma unroll
            for (int r = 0; r < CL; ++r) st_cluster(diag_at[r] + (uint32_t)(k * sizeof(IT)), dv);
    }
    if (xcol) send_columns();
    cluster_sync<CL>(G);

    const float beta_f = __double2float_rn(__ldcg(s.beta + rep));
    int64_t E = __ldcg((const long long *)s.E + rep), bestE = __ldcg((const long long *)s.bestE + rep);
    unsigned long long accepts = 0;
    bool improved = false;

    for (int st = 0; st < s.spe; ++st) {
        const uint32_t step = (uint32_t)(e * s.spe + st);
        const int pb = st & 1;
        int32_t *tgt = s_tgt + pb * npad;
        IT *dlt = s_dlt + pb * npad;

        // ---- 1. proposals of this CTA's locations
        for (int il = warp; il < rows; il += nwarps) {
            const int i = row0 + il;
            const int a = s_phi[i];
            const IT *Ii = sI + (size_t)il * lds;
            const IT Iia = Ii[a];
            const U Dii = (U)(IT)s_Dd[i], Faa = (U)(IT)s_Fd[a];
            const int32_t *Di = s.D + (size_t)i * ldm, *DTi = s.DT + (size_t)i * ldm;
            const int32_t *Fa = s.F + (size_t)a * ldm, *FTa = s.FT + (size_t)a * ldm;
            IT d[8];
            IT mx = (IT)((U)1 << (sizeof(IT) * 8 - 1));     // most negative
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                d[k] = 0;
                const int j = lane + 32 * k;
                if (k < K && j < n) {
                    const int b = s_phi[j];
                    IT Ija;
                    if constexpr (CL == 1) {
                        Ija = sI[j * lds + a];
                    } else {
                        if (j >= row0 && j < row0 + rpc) {
                            Ija = sI[(j - row0) * lds + a];
                        } else if (xcol) {
                            Ija = s_T[il * tld + (j < row0 ? j : j - rpc)];
                        } else {
                            const int r = j / rpc;
                            uint32_t base = I_at[0];
#pragma unroll
                            for (int q = 1; q < CL; ++q) base = (r == q) ? I_at[q] : base;
                            Ija = ld_cluster(base + (uint32_t)(((size_t)(j - r * rpc) * lds + a) * sizeof(IT)), IT(0));
                        }
                    }
                    const int32_t Dij = __ldg(Di + j), Fab = __ldg(Fa + b);
                    const int32_t Dji = SYM ? Dij : __ldg(DTi + j), Fba = SYM ? Fab : __ldg(FTa + b);
                    const U dd = Dii + (U)(IT)s_Dd[j] - (U)(IT)Dij - (U)(IT)Dji;
                    const U ff = Faa + (U)(IT)s_Fd[b] - (U)(IT)Fab - (U)(IT)Fba;
                    d[k] = (IT)((U)Ii[b] + (U)Ija - (U)Iia - (U)s_diag[j] - dd * ff);
                    mx = d[k] > mx ? d[k] : mx;
                }
            }
            mx = warp_max(mx);
            // binary32 weights and the reference's lane-order sums (qap.cu:1069-1110)
            float run = 0.0f, sacc[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                sacc[k] = run;
                if (k < K) {
                    const int j = lane + 32 * k;
                    float w = 0.0f;
                    if (j < n) {
                        const float x = __ll2float_rn((long long)d[k] - (long long)mx);
                        // CUDA's exp2f as the reference writes it (exp2(beta * float(d - max)),
                        // qap.cu:1083-1086), or this library's own 2^x, which the oracle restates
                        w = own_exp2 ? exp2f_neg(__fmul_rn(beta_f, x)) : exp2f(beta_f * x);
                    }
                    run = (k == 0) ? w : __fadd_rn(w, run);
                    sacc[k] = run;
                }
            }
            float x = run;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const float y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x = __fadd_rn(x, y);
            }
            const float off = __fsub_rn(x, run);
            const float total = __shfl_sync(0xffffffffu, __fadd_rn(off, run), 31);
            const float thresh = __fmul_rn(s_uni[il], total);
            int win = -1;
            IT wd = 0, lastd = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int j = lane + 32 * k;
                if (k < K && j < n) {
                    const float cur = __fadd_rn(off, sacc[k]);
                    const float prev = (k == 0) ? off : __fadd_rn(off, sacc[k - 1]);
                    if (cur >= thresh && prev < thresh) {
                        win = j;
                        wd = d[k];
                    }
                    if (j == n - 1) lastd = d[k];
                }
            }
            const unsigned fm = __ballot_sync(0xffffffffu, win >= 0);
            const int src = fm ? __ffs(fm) - 1 : ((n - 1) & 31);   // fallback j = n-1 (:1136-1144)
            const int tj = fm ? __shfl_sync(0xffffffffu, win, src) : n - 1;
            const IT td = __shfl_sync(0xffffffffu, fm ? wd : lastd, src);
            if (lane == 0) {
                if constexpr (CL == 1) {
                    tgt[i] = tj;
                    dlt[i] = td;
                } else {
#pragma unroll
                    for (int r = 0; r < CL; ++r) {
                        st_cluster(tgt_at[r] + (uint32_t)((pb * npad + i) * 4), (int32_t)tj);
                        st_cluster(dlt_at[r] + (uint32_t)((pb * npad + i) * sizeof(IT)), td);
                    }
                }
            }
        }
        cluster_sync<CL>(G);   // every proposal of the replica is in every CTA

        // ---- 2. collisions: a location goes to the best ballot touching it (qap.cu:1150-1225)
        for (int q = tid; q < n; q += BT) s_own[q] = ~0ull;
        draw_thresholds(step + 1u);   // phase 1 of this step has read them (cluster barrier above)
        G.sync();
        for (int q = tid; q < n; q += BT) {
            const int t = tgt[q];
            if (t != q && (unsigned)t < (unsigned)n) {
                const unsigned long long w = oneshot_ballot(dlt[q], q);
                atomicMin(&s_own[t], w);
                atomicMin(&s_own[q], w);
            }
        }
        G.sync();
        int np = 0;
        for (int q0 = 0; q0 < n; q0 += BT) {
            const int q = q0 + tid;
            bool acc = false;
            int t = 0;
            if (q < n) {
                t = tgt[q];
                acc = t != q && (unsigned)t < (unsigned)n && (uint32_t)s_own[q] == (uint32_t)q &&
                      (uint32_t)s_own[t] == (uint32_t)q;
            }
            const unsigned m = __ballot_sync(0xffffffffu, acc);
            if (lane == 0) s_wcnt[warp] = __popc(m);
            G.sync();
            int before = np, all = np;
            for (int w = 0; w < nwarps; ++w) {
                if (w == warp) before = all;
                all += s_wcnt[w];
            }
            if (acc) {
                const int pos = before + __popc(m & ((1u << lane) - 1u));
                s_pi[pos] = q;
                s_pj[pos] = t;
                s_pa[pos] = s_phi[q];
                s_pb[pos] = s_phi[t];
            }
            np = all;
            G.sync();
        }
        // np is the same in every CTA of the cluster; a step without swaps changes nothing
        if (np > 0) {
            for (int p = tid; p < np; p += BT) {                  // qap.cu:1311-1332
                const int i = s_pi[p], j = s_pj[p], a = s_pa[p], b = s_pb[p];
                s_phi[i] = b;
                s_phi[j] = a;
                s_inv[a] = j;
                s_inv[b] = i;
            }

            // ---- 3. force update of this CTA's rows (qap.cu:1337-1412)
            if (tc) {
                // dI = U V^T on the tcgen05 tensor cores: the factors of up to 64 factor columns
                // (swaps, or two columns per swap for asymmetric instances) are staged as fp16
                // MN-major core matrices, A = U over 128 rows (this CTA's, the rest unread), B = V
                // over the columns rounded up to 16; thread 0 issues one M = 128, N = L.tcn,
                // K = 16 MMA per 16 factor columns; the fp32 sums of the whole step accumulate in
                // tensor memory and are added to the rows once.  Exact: every factor is an
                // integer of at most 2048 in magnitude and every sum stays below 2^24 (the host
                // checks both), so fp16 holds the factors and fp32 the sums.
                const uint32_t aS = smem_u32(smem + L.U), bS = aS + (uint32_t)kTcABytes;
                const int kpp = SYM ? 1 : 2, spc = kMmaK / kpp;
                const int ga = (rows + 7) >> 3, gb = (n + 7) >> 3;   // 8-row / 8-column groups
                const uint32_t idesc = umma_idesc_f16_mn(128, L.tcn);
                for (int c0 = 0; c0 < np && !tc_dead; c0 += spc) {
                    const int cn = min(spc, np - c0), kc = cn * kpp, kc16 = (kc + 15) & ~15;
                    // factor column kk of group g: 16 bytes at g * kTcGroupBytes + (kk / 8) * 128 +
                    // (kk % 8) * 16; consecutive threads take consecutive columns, so their
                    // 16-byte stores fill whole core matrices (no bank conflicts).  Column 2p
                    // (or p): D[k][j] - D[k][i] = DT[j][k] - DT[i][k] (doubled when symmetric) and
                    // F[c][b] - F[c][a] = FT[b][c] - FT[a][c]; column 2p + 1: D[j][k] - D[i][k]
                    // and F[b][c] - F[a][c].  Rows are read in 16-byte pieces up to rpc (D) and
                    // npad (F), within the zero-padded ldm.
                    for (int idx = tid; idx < (ga + gb) * kc; idx += BT) {
                        const int grp = idx / kc, kk = idx - grp * kc;
                        const int p = c0 + kk / kpp, part = SYM ? 0 : (kk & 1);
                        const bool isA = grp < ga;
                        const int gg = isA ? grp : grp - ga;
                        const int x = isA ? s_pi[p] : s_pa[p], y = isA ? s_pj[p] : s_pb[p];
                        const int32_t *M = isA ? (part ? s.D : s.DT) : (part ? s.F : s.FT);
                        const int off = (isA ? row0 : 0) + 8 * gg, lim = isA ? rpc : npad;
                        const int4 *hp = reinterpret_cast<const int4 *>(M + (size_t)y * ldm + off);
                        const int4 *lp = reinterpret_cast<const int4 *>(M + (size_t)x * ldm + off);
                        const int4 z = make_int4(0, 0, 0, 0);
                        const int4 h0 = __ldg(hp), l0 = __ldg(lp);
                        const bool two = 8 * gg + 4 < lim;
                        const int4 h1 = two ? __ldg(hp + 1) : z, l1 = two ? __ldg(lp + 1) : z;
                        const uint4 w = pack_half8(h0, l0, h1, l1, (SYM && isA) ? 2 : 1);
                        *reinterpret_cast<uint4 *>(smem + L.U + (isA ? 0 : kTcABytes) + (size_t)gg * kTcGroupBytes +
                                                   (kk >> 3) * 128 + (kk & 7) * 16) = w;
                    }
                    // zero factor columns kc..kc16-1, which the last K = 16 step reads
                    for (int idx = tid; idx < (ga + gb) * (kc16 - kc); idx += BT) {
                        const int grp = idx / (kc16 - kc), kk = kc + idx - grp * (kc16 - kc);
                        const bool isA = grp < ga;
                        const int gg = isA ? grp : grp - ga;
                        *reinterpret_cast<uint4 *>(smem + L.U + (isA ? 0 : kTcABytes) + (size_t)gg * kTcGroupBytes +
                                                   (kk >> 3) * 128 + (kk & 7) * 16) = make_uint4(0u, 0u, 0u, 0u);
                    }
                    fence_async_smem();
                    G.sync();                                // the chunk's factors are staged
                    if (tid == 0) {
                        tc_fence_after();
                        for (int ks = 0; ks < kc16 / 16; ++ks)
                            umma_f16(tmem, umma_desc_mn(aS + 256u * ks, 128u, kTcGroupBytes),
                                     umma_desc_mn(bS + 256u * ks, 128u, kTcGroupBytes), idesc, c0 > 0 || ks > 0);
                        umma_commit(tc_bar);
                    }
                    // the MMAs have read the factors (the next chunk may restage them) and their
                    // sums are in tensor memory
                    const bool gave_up = !mbar_wait_bounded(tc_bar, tc_phase, kWaitLimitNs);
                    tc_phase ^= 1u;
                    if (G.sync_or(gave_up)) {
                        if (tid == 0) atomicOr(s.error, kErrTimeout);
                        tc_dead = true;
                    }
                }
                if (!tc_dead) {
                    // warp w reads TMEM lanes 32 (w % 4) .. + 31 (rows), 16 columns at a time, the
                    // column blocks spread over the warps of each lane quarter
                    tc_fence_after();
                    const int quad = warp & 3, r = 32 * quad + lane;
                    for (int cb = warp >> 2; 16 * cb < L.tcn; cb += nwarps >> 2) {
                        uint32_t v[16];
                        tmem_ld16(tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)(16 * cb), v);
                        tmem_wait_ld();
                        if (r < rows) {
                            IT *dst = sI + (size_t)r * lds + 16 * cb;
#pragma unroll
                            for (int t = 0; t < 16; ++t)
                                if (16 * cb + t < n) dst[t] = (IT)((U)dst[t] + (U)(IT)__float2int_rn(__uint_as_float(v[t])));
                        }
                    }
                    tc_fence_before();                       // before the next step's MMAs overwrite
                }
                G.sync();
            } else if (mma) {
                // dI = U^T V on the tensor cores (m16n8k16, fp16 in, fp32 sums): the factors are
                // integers of at most 2048 in magnitude and every sum stays below 2^24 (the host
                // checks both), so the products and sums are exact; added to the rows once
                __half *hU = reinterpret_cast<__half *>(smem + L.U);
                const int rb16 = (rpc + 15) & ~15, nc8 = (n + 7) & ~7;
                __half *hV = hU + (size_t)rb16 * kMmaLd;
                const int kpp = SYM ? 1 : 2;                 // factor columns per swap
                const int spc = kMmaK / kpp;                 // swaps per staged chunk
                const int nrb = (rows + 15) >> 4, nct = (n + 7) >> 3;
                const int ngroups = nrb * ((nct + 7) >> 3);  // 16 x 64 output blocks
                const int g8 = lane >> 2, t4 = lane & 3;
                // chunk by chunk: stage the factors once, then every warp runs its 16 x 64 output
                // blocks and adds each block's sums (below 2^24, exact) to the rows
                for (int c0 = 0; c0 < np; c0 += spc) {
                    const int cn = min(spc, np - c0), kc = cn * kpp;
                    // U[k][col]: 2 (D[k][j] - D[k][i]) (symmetric) or D[k][j] - D[k][i] and
                    // D[j][k] - D[i][k]; V[c][col]: F[c][b] - F[c][a] (and F[b][c] - F[a][c])
                    // consecutive threads take consecutive swaps of one row group, so their
                    // 2-byte stores into a factor row are conflict-free
#pragma unroll 2
                    for (int idx = tid; idx < cn * (rpc >> 2); idx += BT) {
                        const int q4 = idx / cn, p = idx - q4 * cn;
                        const int i = s_pi[c0 + p], j = s_pj[c0 + p];
                        const int4 hi = __ldg(reinterpret_cast<const int4 *>(s.DT + (size_t)j * ldm + row0) + q4);
                        const int4 lo = __ldg(reinterpret_cast<const int4 *>(s.DT + (size_t)i * ldm + row0) + q4);
                        const int h4[4] = {hi.x - lo.x, hi.y - lo.y, hi.z - lo.z, hi.w - lo.w};
#pragma unroll
                        for (int r = 0; r < 4; ++r)
                            hU[(size_t)(4 * q4 + r) * kMmaLd + p * kpp] = __int2half_rn(SYM ? 2 * h4[r] : h4[r]);
                        if constexpr (!SYM) {
                            const int4 hi2 = __ldg(reinterpret_cast<const int4 *>(s.D + (size_t)j * ldm + row0) + q4);
                            const int4 lo2 = __ldg(reinterpret_cast<const int4 *>(s.D + (size_t)i * ldm + row0) + q4);
                            const int d4[4] = {hi2.x - lo2.x, hi2.y - lo2.y, hi2.z - lo2.z, hi2.w - lo2.w};
#pragma unroll
                            for (int r = 0; r < 4; ++r)
                                hU[(size_t)(4 * q4 + r) * kMmaLd + p * kpp + 1] = __int2half_rn(d4[r]);
                        }
                    }
#pragma unroll 2
                    for (int idx = tid; idx < cn * (npad >> 2); idx += BT) {
                        const int q4 = idx / cn, p = idx - q4 * cn;
                        const int a = s_pa[c0 + p], b = s_pb[c0 + p];
                        const int4 hi = __ldg(reinterpret_cast<const int4 *>(s.FT + (size_t)b * ldm) + q4);
                        const int4 lo = __ldg(reinterpret_cast<const int4 *>(s.FT + (size_t)a * ldm) + q4);
                        const int h4[4] = {hi.x - lo.x, hi.y - lo.y, hi.z - lo.z, hi.w - lo.w};
#pragma unroll
                        for (int r = 0; r < 4; ++r) hV[(size_t)(4 * q4 + r) * kMmaLd + p * kpp] = __int2half_rn(h4[r]);
                        if constexpr (!SYM) {
                            const int4 hi2 = __ldg(reinterpret_cast<const int4 *>(s.F + (size_t)b * ldm) + q4);
                            const int4 lo2 = __ldg(reinterpret_cast<const int4 *>(s.F + (size_t)a * ldm) + q4);
                            const int d4[4] = {hi2.x - lo2.x, hi2.y - lo2.y, hi2.z - lo2.z, hi2.w - lo2.w};
#pragma unroll
                            for (int r = 0; r < 4; ++r) hV[(size_t)(4 * q4 + r) * kMmaLd + p * kpp + 1] = __int2half_rn(d4[r]);
                        }
                    }
                    // zeros in the factor columns kc..(kc rounded up to 16)-1 that the last
                    // k-step reads (the space held other data); padded rows and columns
                    // only reach output entries that are never written back
                    const int kz = ((kc + 15) & ~15) - kc;
                    for (int idx = tid; idx < (rpc + npad) * kz; idx += BT) {
                        const int row = idx / kz, kk = kc + idx - row * kz;
                        if (row < rpc) hU[(size_t)row * kMmaLd + kk] = __int2half_rn(0);
                        else hV[(size_t)(row - rpc) * kMmaLd + kk] = __int2half_rn(0);
                    }
                    G.sync();
                    for (int blk = warp; blk < ngroups; blk += nwarps) {
                        const int rb = blk % nrb, cg = blk / nrb;
                        float acc[8][4];
#pragma unroll
                        for (int t8 = 0; t8 < 8; ++t8)
#pragma unroll
                            for (int q = 0; q < 4; ++q) acc[t8][q] = 0.0f;
                        for (int ks = 0; ks * 16 < kc; ++ks) {
                            const __half *ar = hU + (size_t)(rb * 16 + g8) * kMmaLd + ks * 16 + 2 * t4;
                            uint32_t af[4];
                            af[0] = *reinterpret_cast<const uint32_t *>(ar);
                            af[1] = *reinterpret_cast<const uint32_t *>(ar + 8 * kMmaLd);
                            af[2] = *reinterpret_cast<const uint32_t *>(ar + 8);
                            af[3] = *reinterpret_cast<const uint32_t *>(ar + 8 * kMmaLd + 8);
#pragma unroll
                            for (int t8 = 0; t8 < 8; ++t8) {
                                const int ct = cg * 8 + t8;
                                if (ct < nct) {
                                    const __half *br = hV + (size_t)(ct * 8 + g8) * kMmaLd + ks * 16 + 2 * t4;
                                    uint32_t bf[2];
                                    bf[0] = *reinterpret_cast<const uint32_t *>(br);
                                    bf[1] = *reinterpret_cast<const uint32_t *>(br + 8);
                                    mma_16816(acc[t8], af, bf);
                                }
                            }
                        }
#pragma unroll
                        for (int t8 = 0; t8 < 8; ++t8) {
                            const int c = (cg * 8 + t8) * 8 + 2 * t4;
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                const int r = rb * 16 + g8 + (q >> 1) * 8, cc = c + (q & 1);
                                if (r < rows && cc < n) {
                                    IT *dst = sI + (size_t)r * lds + cc;
                                    *dst = (IT)((U)*dst + (U)(IT)(long long)acc[t8][q]);
                                }
                            }
                        }
                    }
                    G.sync();                                // before the next chunk is staged
                }
                G.sync();
            } else {
                for (int c0 = 0; c0 < np; c0 += pc) {
                    const int cn = min(pc, np - c0);
                    // the chunk's factors from 16-byte row pieces of D^T, D, F^T, F, several pieces
                    // per thread in flight (rows are zero padded to ldm >= cl * rpc, npad)
                    constexpr int UNR = SYM ? 4 : 2;   // 512 threads: 128 registers each
                    stage_factors<IT, SYM, SYM, UNR>(tid, BT, cn, rpc / 4, s.DT + row0, s.D + row0, ldm, s_pi + c0, s_pj + c0,
                                           s_U, s_U2, rpc);
                    stage_factors<IT, SYM, false, UNR>(tid, BT, cn, npad / 4, s.FT, s.F, ldm, s_pa + c0, s_pb + c0, s_V, s_V2,
                                           vld);
                    for (int idx = tid; idx < cn * (vld - npad); idx += BT) {   // columns npad..vld-1
                        const int p = idx / (vld - npad), c = npad + idx - p * (vld - npad);
                        s_V[p * vld + c] = 0;
                        if constexpr (!SYM) s_V2[p * vld + c] = 0;
                    }
                    G.sync();
                    for (int kq = warp * RT; kq < rows; kq += nwarps * RT) {
                        U acc[RT][8];
#pragma unroll
                        for (int r = 0; r < RT; ++r)
#pragma unroll
                            for (int q = 0; q < 8; ++q) {
                                const int c = lane + 32 * q;
                                acc[r][q] = (q < K && c < n && kq + r < rows) ? (U)sI[(size_t)(kq + r) * lds + c] : (U)0;
                            }
                        {   // U / V rows are padded (rpc, 256 entries), so no load needs a guard
                            const uint32_t ua = smem_u32(s_U) + (uint32_t)(kq * sizeof(IT));
                            const uint32_t va = smem_u32(s_V) + (uint32_t)(lane * sizeof(IT));
                            const uint32_t ua2 = smem_u32(s_U2) + (uint32_t)(kq * sizeof(IT));
                            const uint32_t va2 = smem_u32(s_V2) + (uint32_t)(lane * sizeof(IT));
                            for (int p = 0; p < cn; ++p) {
                                U uu[RT], vv[8];
#pragma unroll
                                for (int r = 0; r < RT; ++r) uu[r] = (U)lds_it<IT>(ua + (uint32_t)((p * rpc + r) * sizeof(IT)));
#pragma unroll
                                for (int q = 0; q < 8; ++q) vv[q] = (U)lds_it<IT>(va + (uint32_t)((p * 256 + 32 * q) * sizeof(IT)));
#pragma unroll
                                for (int r = 0; r < RT; ++r)
#pragma unroll
                                    for (int q = 0; q < 8; ++q) acc[r][q] += uu[r] * vv[q];
                                if constexpr (!SYM) {
#pragma unroll
                                    for (int r = 0; r < RT; ++r) uu[r] = (U)lds_it<IT>(ua2 + (uint32_t)((p * rpc + r) * sizeof(IT)));
#pragma unroll
                                    for (int q = 0; q < 8; ++q) vv[q] = (U)lds_it<IT>(va2 + (uint32_t)((p * 256 + 32 * q) * sizeof(IT)));
#pragma unroll
                                    for (int r = 0; r < RT; ++r)
#pragma unroll
                                        for (int q = 0; q < 8; ++q) acc[r][q] += uu[r] * vv[q];
                                }
                            }
                        }
#pragma unroll
                        for (int r = 0; r < RT; ++r)
#pragma unroll
                            for (int q = 0; q < 8; ++q) {
                                const int c = lane + 32 * q;
                                if (q < K && c < n && kq + r < rows) sI[(size_t)(kq + r) * lds + c] = (IT)acc[r][q];
                            }
                    }
                    G.sync();
                }

            }

            // ---- 4. new diagonal and energy (qap.cu:1420-1458): E = -1/2 sum_k I[k][phi(k)]
            long long mys = 0;
            for (int kk = tid; kk < rows; kk += BT) {
                const int k = row0 + kk;
                const IT dv = sI[(size_t)kk * lds + s_phi[k]];
                mys += (long long)dv;
                if constexpr (CL == 1) s_diag[k] = dv;
                else
#pragma unroll
                    for (int r = 0; r < CL; ++r) st_cluster(diag_at[r] + (uint32_t)(k * sizeof(IT)), dv);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) mys += __shfl_xor_sync(0xffffffffu, mys, o);
            if (lane == 0) s_part[CL + warp] = mys;
            G.sync();
            if (tid == 0) {
                long long t = 0;
                for (int w = 0; w < nwarps; ++w) t += s_part[CL + w];
                if constexpr (CL == 1) s_part[0] = t;
                else
#pragma unroll
                    for (int r = 0; r < CL; ++r) st_cluster(part_at[r] + (uint32_t)(rank * 8), (int64_t)t);
            }
            cluster_sync<CL>(G);   // new rows, diagonal and energy shares everywhere
            long long tot = 0;
#pragma unroll
            for (int r = 0; r < CL; ++r) tot += s_part[r];
            E = -tot / 2;
            accepts += (unsigned long long)np;
            if (xcol) {   // every CTA is past its force update: T (over U / V) may be written
                send_columns();
                cluster_sync<CL>(G);
            }
        }
        if (E < bestE) {
            bestE = E;
            improved = true;
            if (rank == 0) {
                for (int q = tid; q < n; q += BT) s_bphi[q] = s_phi[q];
                if constexpr (GP) {
                    if (E < s.ev.goal_print) {
                        if (tid == 0) s_flag[0] = goal_print_claim(s.ev, g, l, e, E);
                        G.sync();
                        const int slot = s_flag[0];
                        if (slot >= 0)
                            for (int q = tid; q < n; q += BT) s.ev.perm[(size_t)slot * n + q] = s_phi[q];
                    }
                }
            }
        }
    }

    // ---- store the replica
    cluster_sync<CL>(G);   // no CTA reads another's shared memory any more
    if (tc) {   // every tensor-memory read has completed (tcgen05.wait::ld, fence, barrier)
        if (warp == 0) {
            // after a wait that gave up, one more bounded wait for the MMAs still in flight
            if (tc_dead) mbar_wait_bounded(tc_bar, tc_phase ^ 1u, kWaitLimitNs);
            tc_fence_after();
            tmem_dealloc(tmem, (uint32_t)L.tcols);
        }
        if (tid == 0) mbar_inval(tc_bar);
    }
    {
        IT *gI = reinterpret_cast<IT *>(s.I) + ((size_t)rep * n + row0) * s.ldg;
        const int nvg = s.ldg / VEC;
        for (int idx = tid; idx < rows * nvg; idx += BT) {
            const int k = idx / nvg, v = idx - k * nvg;
            Vec<IT> w;
#pragma unroll
            for (int q = 0; q < VEC; ++q) w.v[q] = sI[(size_t)k * lds + v * VEC + q];
            *reinterpret_cast<Vec<IT> *>(gI + (size_t)k * s.ldg + v * VEC) = w;
        }
    }
    if (rank == 0) {
        int32_t *gphi = s.phi + (size_t)rep * n;
        for (int q = tid; q < n; q += BT) gphi[q] = s_phi[q];
        if (improved) {
            int32_t *gb = s.best_phi + (size_t)rep * n;
            for (int q = tid; q < n; q += BT) gb[q] = s_bphi[q];
        }
        if (tid == 0) {
            s.E[rep] = E;
            s.bestE[rep] = bestE;
            s.accepts[rep] = __ldcg(s.accepts + rep) + accepts;
        }
    }
    __threadfence();
    return true;
}

// Solve path: one launch = one epoch of every replica of the solve (grid = T*R*CL CTAs);
// the last replica of each group to finish runs the group's tracking + exchange.
// KIND: 0 the generic sequential epoch, 1 the binary-flow one, 2 the one-shot epoch (up to
// 512 threads: its proposals are independent, so more warps hide more latency).
template <class IT, int CL, bool SYM, bool GP, int KIND = 0>
__global__ void __launch_bounds__(KIND == 2 ? 512 : 256, (CL == 4 && KIND != 2) ? 2 : 1) epoch_kernel(SolveDev s) {
    extern __shared__ __align__(16) unsigned char smem[];
    int rank = 0;
    if constexpr (CL > 1) rank = (int)cg::this_cluster().block_rank();
    const int rep = blockIdx.x / CL;
    const int g = rep / s.R;
    // Every CTA of a group reads the same epoch and stop values: stop_epoch only drops to
    // epoch+1 during this launch, so the test below cannot differ inside a cluster or group.
    const int e = *((volatile int32_t *)s.epoch + g);
    if (e >= *(volatile int32_t *)s.stop_epoch) return;
    const Grp G{(int)threadIdx.x, (int)blockDim.x, (int)(threadIdx.x & 31), (int)(threadIdx.x >> 5),
                (int)(blockDim.x >> 5), 0};
    bool ok;
    if constexpr (KIND == 1) ok = replica_epoch_bin<CL>(s, rep, rank, e, G, smem);
    else if constexpr (KIND == 2) ok = replica_epoch_os<IT, CL, SYM, GP>(s, rep, rank, e, G, smem);
    else if constexpr (KIND == 3) ok = replica_epoch_pipe<CL>(s, rep, rank, e, smem);
    else ok = replica_epoch<IT, CL, SYM, GP>(s, rep, rank, e, G, smem);
    __syncthreads();
    if (ok && rank == 0 && threadIdx.x == 0) {
        const unsigned prev = atomicAdd(s.finish + g, 1u);
        if (prev == (unsigned)s.R - 1u) {
            __threadfence();
            track_exchange(s, g, e + 1, smem);   // the epoch's shared memory is dead now
            s.finish[g] = 0u;
            s.epoch[g] = e + 1;
            __threadfence();
        }
    }
}

// The paired binary-flow epoch: cluster c of CL CTAs runs replicas 2c and 2c + 1, each on half
// of every CTA's warps (named barriers 1 and 2) over one shared copy of the instance tables.
// Both halves take part in the two cluster barriers of an epoch whether or not their replica
// runs (an odd replica count leaves the last half idle; a group past its stop epoch idles).
template <int CL>
__global__ void __launch_bounds__(512, 1) epoch_pair_kernel(SolveDev s) {
    extern __shared__ __align__(16) unsigned char smem[];
    int rank = 0;
    if constexpr (CL > 1) rank = (int)cg::this_cluster().block_rank();
    const BinPairLayout P(s.n, s.rpc, s.lds, CL);
    int16_t *Ds = reinterpret_cast<int16_t *>(smem + P.Ds);
    uint32_t *Fb = reinterpret_cast<uint32_t *>(smem + P.Fb);
    load_bin_instance(s, rank, (int)threadIdx.x, (int)blockDim.x, (int)(threadIdx.x & 31),
                      (int)(threadIdx.x >> 5), (int)(blockDim.x >> 5), Ds, Fb);
    __syncthreads();
    const int half_threads = (int)blockDim.x / 2;
    const int h = (int)threadIdx.x / half_threads;
    const int tid = (int)threadIdx.x - h * half_threads;
    const Grp G{tid, half_threads, tid & 31, tid >> 5, half_threads >> 5, 1 + h};
    const int rep = 2 * ((int)blockIdx.x / CL) + h;
    bool run = rep < s.T * s.R;
    int g = 0, e = 0;
    if (run) {
        g = rep / s.R;
        e = *((volatile int32_t *)s.epoch + g);
        run = e < *(volatile int32_t *)s.stop_epoch;
    }
    if (!run) {   // the cluster barriers of an epoch, without a replica
        cluster_sync<CL>(G);
        cluster_sync<CL>(G);
        return;
    }
    const bool ok = replica_epoch_bin<CL>(s, rep, rank, e, G, smem + P.rep[h], Ds, Fb);
    G.sync();
    if (ok && rank == 0 && tid == 0) {
        const unsigned prev = atomicAdd(s.finish + g, 1u);
        if (prev == (unsigned)s.R - 1u) {
            __threadfence();
            track_exchange(s, g, e + 1, smem + P.rep[h]);   // this half's section is dead now
            s.finish[g] = 0u;
            s.epoch[g] = e + 1;
            __threadfence();
        }
    }
}

// The persistent solve: CTA (cluster) rep / CL runs replica rep for every mega-iteration of the
// launch, from *epoch_all up to *run_end.  After each epoch the last replica of a group runs the
// group's tracking + exchange, the last group releases the next mega-iteration (*epoch_all) and,
// when the host's kill word is set, moves the stop to the next boundary.  Thread 0 of the
// cluster's rank 0 waits for the release (bounded) and decides whether the cluster goes on; the
// decision reaches the cluster's other CTAs through rank 0's shared memory between two cluster
// barriers, so a cluster never splits.  A kernel boundary of the per-epoch launches and this
// barrier order the same steps, so both take the same trajectory.  Needs every CTA resident.
template <class IT, int CL, bool SYM, bool GP, int KIND>
__global__ void __launch_bounds__(KIND == 2 ? 512 : 256, (CL == 4 && KIND != 2) ? 2 : 1) solve_kernel(SolveDev s) {
    // Between epochs no shared memory is live: the first word carries the cluster's decision.
    extern __shared__ __align__(16) unsigned char smem[];
    volatile int32_t *s_go = reinterpret_cast<volatile int32_t *>(smem);
    int rank = 0;
    if constexpr (CL > 1) rank = (int)cg::this_cluster().block_rank();
    const int rep = blockIdx.x / CL;
    const int g = rep / s.R;
    const Grp G{(int)threadIdx.x, (int)blockDim.x, (int)(threadIdx.x & 31), (int)(threadIdx.x >> 5),
                (int)(blockDim.x >> 5), 0};
    volatile int32_t *epoch_all = s.epoch_all;
    int e = -1;                                   // the epoch just run (-1: none yet)
    unsigned long long spent = 0;                 // its duration
    for (;;) {
        if (rank == 0 && threadIdx.x == 0) {
            bool released = true;
            if (e >= 0) {
                // the slowest replica takes about as long as this one: a healthy wait is a fraction
                // of an epoch, so the limit is eight epochs of this replica and at least two seconds
                const unsigned long long limit = max(2000000000ull, 8ull * spent);
                const unsigned long long w0 = globaltimer_ns();
                while (*epoch_all <= e) {
                    if (*(volatile int32_t *)s.error != 0) {
                        released = false;
                        break;
                    }
                    if (globaltimer_ns() - w0 > limit) {
                        atomicOr(s.error, kErrTimeout);
                        released = false;
                        break;
                    }
                }
                __threadfence();
            }
            const int en = *epoch_all;
            const int stop = min(*(volatile int32_t *)s.stop_epoch, *(volatile const int32_t *)s.run_end);
            *s_go = (released && en < stop && *(volatile int32_t *)s.error == 0) ? en : -1;
        }
        if constexpr (CL > 1) {
            cluster_barrier<CL>();
            int go;
            asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(go) : "r"(cluster_addr(smem_u32(smem), 0)) : "memory");
            e = go;
            cluster_barrier<CL>();                // every CTA has read it before rank 0 reuses the word
        } else {
            __syncthreads();
            e = *s_go;
            __syncthreads();
        }
        if (e < 0) break;
        const unsigned long long t0 = globaltimer_ns();
        bool ok;
        if constexpr (KIND == 1) ok = replica_epoch_bin<CL>(s, rep, rank, e, G, smem);
        else if constexpr (KIND == 2) ok = replica_epoch_os<IT, CL, SYM, GP>(s, rep, rank, e, G, smem);
        else ok = replica_epoch<IT, CL, SYM, GP>(s, rep, rank, e, G, smem);
        __syncthreads();
        spent = globaltimer_ns() - t0;
        // a failed epoch has set the error word; rank 0 sees it while it waits and stops the cluster
        if (ok && rank == 0 && threadIdx.x == 0 && atomicAdd(s.finish + g, 1u) == (unsigned)s.R - 1u) {
            __threadfence();
            // the epoch's shared memory is dead; the decision word at offset 0 is written only
            // after the release, past the scratch's use
            track_exchange(s, g, e + 1, smem + 16);
            s.finish[g] = 0u;
            s.epoch[g] = e + 1;
            __threadfence();
            if (s.T == 1 || atomicAdd(s.finish_all, 1u) == (unsigned)s.T - 1u) {
                *s.finish_all = 0u;
                if (s.kill && *s.kill) atomicMin(s.stop_epoch, e + 1);
                __threadfence();
                *epoch_all = e + 1;               // release mega-iteration e + 1
            }
        }
    }
}

// ------------------------------------------------------------------ the batch kernel

constexpr unsigned long long kQueueWaitNs = 30000000000ull;   // 30 s without any progress
constexpr unsigned long long kDoneItem = ~0ull;

// An instance descriptor read through L2.  A serving launch rewrites descriptors while it
// runs (a slot is reused by the next request), and another SM's L1 may still hold the old
// lines, so device code never reads B.inst[k] (nor B.sym / B.max_megaiters) through L1.
// (The words are assembled in a word array and copied into the struct with memcpy: storing
// them through an unsigned long long pointer into a SolveDev would break type-based aliasing,
// and the compiler may then read the fields before or without those stores.)
__device__ __forceinline__ void load_desc(SolveDev &d, const SolveDev *p) {
    constexpr int kWords = (int)(sizeof(SolveDev) / 8);
    static_assert(sizeof(SolveDev) % 8 == 0, "descriptor copied in 8-byte words");
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(p);
    unsigned long long w[kWords];
#pragma unroll
    for (int q = 0; q < kWords; ++q) w[q] = __ldcg(src + q);
    memcpy(&d, w, sizeof(SolveDev));
}

// Enqueues every replica of instance k for its next epoch.
__device__ void queue_push_instance(const BatchDev &B, int k, int replicas) {
    const unsigned long long base = atomicAdd(B.q_tail, (unsigned long long)replicas);
    for (int q = 0; q < replicas; ++q)
        B.q_items[(unsigned)(base + q) & B.qmask] = ((unsigned long long)k << 32) | (unsigned)q;
    __threadfence();
    for (int q = 0; q < replicas; ++q)
        *((volatile unsigned long long *)B.q_seq + ((unsigned)(base + q) & B.qmask)) = base + q + 1;
}

constexpr unsigned long long kAdmitItem = 1ull << 63;   // a serving admission, not a queue item
constexpr unsigned long long kNoTicket = ~0ull;

__device__ void set_error(const BatchDev &B, int32_t bits) {
    const int32_t old = atomicOr(B.error, bits);
    if (B.serving) {
        *B.link.error_host = old | bits;
        __threadfence_system();
    }
}

// Serving: claims one request the host has published (returns its inbox entry, or 0).
__device__ unsigned long long inbox_claim(const BatchDev &B) {
    const unsigned long long h = *(volatile unsigned long long *)B.link.inbox_head;
    if (h >= *B.link.inbox_tail) return 0;
    if (atomicCAS(B.link.inbox_head, h, h + 1) != h) return 0;
    __threadfence_system();
    return B.link.inbox[h & B.link.inbox_mask] | kAdmitItem;
}

// Serving: reports a finished instance to the host.
__device__ void report_done(const BatchDev &B, int k) {
    const unsigned long long idx = atomicAdd(B.link.done_tail, 1ull);
    B.link.done[idx & B.link.done_mask] = (unsigned long long)k;
    __threadfence_system();
    B.link.done_seq[idx & B.link.done_mask] = idx + 1;
    __threadfence_system();
}

// Serving: the finished instance's result, best permutation and final energies, written into
// its mapped result slot (one thread).
__device__ void publish_result(const BatchDev &B, int k) {
    SolveDev s;
    load_desc(s, B.inst + k);
    const int reps = s.T * s.R;
    long long best = 0x7fffffffffffffffll, arg = 0;
    unsigned long long acc = 0;
    for (int r = 0; r < reps; ++r) {
        const long long v = __ldcg((const long long *)s.bestE + r);
        if (v < best) { best = v; arg = r; }
        acc += __ldcg(s.accepts + r);
    }
    volatile BatchResultDev &o = B.link.results[k];
    o.best = best;
    o.arg = arg;
    o.accepts = acc;
    o.single_best = __ldcg((const long long *)s.single_best);
    o.target_epoch = __ldcg((const long long *)s.target_epoch);
    o.target_ns = __ldcg(s.target_ns);
    o.epoch = __ldcg(s.epoch);
    o.stop_epoch = __ldcg(s.stop_epoch);
    o.error = __ldcg(s.error);
    for (int q = 0; q < s.n; ++q) B.link.result_perm[(size_t)k * kMaxN + q] = __ldcg(s.best_phi + arg * s.n + q);
    for (int r = 0; r < reps && r < B.link.energy_stride; ++r)
        B.link.result_energy[(size_t)k * B.link.energy_stride + r] = __ldcg((const long long *)s.E + r);
    __threadfence_system();
}

// Next item for a worker that holds queue ticket `ticket` (taken when it holds none): the
// ticket's item, a serving admission (the ticket is kept), or kDoneItem once no instance is
// running and shutdown is set.  A batch's wait is bounded (its items come from workers that
// are finishing epochs); a serving launch waits while the host's heartbeat advances.
__device__ unsigned long long queue_next(const BatchDev &B, unsigned long long &ticket) {
    if (ticket == kNoTicket) ticket = atomicAdd(B.q_head, 1ull);
    const unsigned slot = (unsigned)ticket & B.qmask;
    unsigned long long t0 = globaltimer_ns();
    unsigned long long beat = B.serving ? *B.link.heartbeat : 0;
    for (;;) {
        const int32_t sd = *B.shutdown;   // 1: drain, then leave; 2: leave now
        if (sd == 2) return kDoneItem;    // even with work queued (the host abandons it)
        if (*((volatile unsigned long long *)B.q_seq + slot) == ticket + 1) {
            __threadfence();
            ticket = kNoTicket;
            return *((volatile unsigned long long *)B.q_items + slot);
        }
        if (sd != 0 && *(volatile int32_t *)B.active == 0) return kDoneItem;
        if (B.serving) {
            const unsigned long long adm = inbox_claim(B);
            if (adm) return adm;
            const unsigned long long now_beat = *B.link.heartbeat;
            const unsigned long long now = globaltimer_ns();
            if (now_beat != beat) {
                beat = now_beat;
                t0 = now;
            } else if (now - t0 > B.link.heartbeat_limit_ns) {
                set_error(B, kErrHostLost);
                return kDoneItem;
            }
            __nanosleep(1000);
        } else {
            if (globaltimer_ns() - t0 > kQueueWaitNs) {
                set_error(B, kErrTimeout);
                return kDoneItem;
            }
            __nanosleep(200);
        }
    }
}

// Serving admission by a whole worker: the descriptor into the device table, the head image
// from mapped memory into the instance's device head, the tail cleared; then one set-up item
// per replica is queued.
__device__ void serve_admit(const BatchDev &B, unsigned long long entry, const Grp &G) {
    const int slot = (int)((entry >> 32) & 0x7fffffffull);
    const int stg = (int)(entry & 0xffffffffull);
    const volatile ServeDesc &d = B.link.desc[slot];
    char *head = (char *)d.dev.D;            // the head region starts with D (carve order)
    char *tail = (char *)d.dev.I;            // the tail region starts with I
    const unsigned long long hb = d.head_bytes, tb = d.tail_bytes;
    // The staging buffers are mapped host memory that the host refills for the next request:
    // read them uncached (ld.global.cv), or this SM's L1 could return the previous request's
    // image of the same buffer.
    const int4 *src = reinterpret_cast<const int4 *>(B.link.staging + (size_t)stg * B.link.staging_stride);
    for (unsigned long long q = G.tid; q < hb / 16; q += G.BT) reinterpret_cast<int4 *>(head)[q] = __ldcv(src + q);
    const int4 z = make_int4(0, 0, 0, 0);
    for (unsigned long long q = G.tid; q < tb / 16; q += G.BT) reinterpret_cast<int4 *>(tail)[q] = z;
    if (G.tid == 0) {
        const volatile unsigned long long *dw = reinterpret_cast<const volatile unsigned long long *>(&d.dev);
        unsigned long long *iw = reinterpret_cast<unsigned long long *>(B.link.inst_rw + slot);
        for (int q = 0; q < (int)(sizeof(SolveDev) / 8); ++q) iw[q] = dw[q];
        B.link.sym_rw[slot] = d.sym;
        B.link.maxm_rw[slot] = d.max_megaiters;
    }
    __threadfence();
    G.sync();
    if (G.tid == 0) {
        B.link.staging_busy[stg] = 0;         // the host may reuse the staging buffer
        __threadfence_system();
        SolveDev s;
        load_desc(s, B.inst + slot);
        atomicAdd(B.active, 1);
        const int replicas = s.T * s.R;
        const unsigned long long base = atomicAdd(B.q_tail, (unsigned long long)replicas);
        for (int q = 0; q < replicas; ++q)
            B.q_items[(unsigned)(base + q) & B.qmask] =
                ((unsigned long long)slot << 32) | (unsigned)q | (unsigned long long)kSetupItem;
        __threadfence();
        for (int q = 0; q < replicas; ++q)
            *((volatile unsigned long long *)B.q_seq + ((unsigned)(base + q) & B.qmask)) = base + q + 1;
    }
    G.sync();
}

// setup() of one served replica on the device (CPU_PIM.cpp:164-192): force matrix from its
// permutation, energy = -1/2 sum_i I[i][phi(i)], best energy unset.  `sphi` is a shared
// scratch of n ints, `sred` of one long long per warp.
template <class IT>
__device__ void replica_setup(const SolveDev &s, int rep, const Grp &G, int32_t *sphi, long long *sred) {
    const int n = s.n, ldg = s.ldg, ldm = s.ldm;
    const int32_t *phi = s.phi + (size_t)rep * n;
    for (int q = G.tid; q < n; q += G.BT) {
        const int p = __ldcg(phi + q);
        sphi[q] = p;
        s.best_phi[(size_t)rep * n + q] = p;
    }
    G.sync();
    IT *I = reinterpret_cast<IT *>(s.I) + (size_t)rep * n * ldg;
    for (int idx = G.tid; idx < n * ldg; idx += G.BT) {
        const int i = idx / ldg, a = idx - i * ldg;
        long long acc = 0;
        if (a < n) {
            const int32_t *Di = s.D + (size_t)i * ldm, *DTi = s.DT + (size_t)i * ldm;
            const int32_t *Fa = s.F + (size_t)a * ldm, *FTa = s.FT + (size_t)a * ldm;
            for (int j = 0; j < n; ++j) {
                const int pj = sphi[j];
                acc += (long long)__ldcg(Di + j) * __ldcg(Fa + pj) + (long long)__ldcg(DTi + j) * __ldcg(FTa + pj);
            }
        }
        I[(size_t)i * ldg + a] = (IT)(-acc);
    }
    __threadfence();
    G.sync();
    long long e = 0;
    for (int i = G.tid; i < n; i += G.BT) e += (long long)__ldcg(I + (size_t)i * ldg + sphi[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    if (G.lane == 0) sred[G.warp] = e;
    G.sync();
    if (G.tid == 0) {
        long long t = 0;
        for (int w = 0; w < G.nwarps; ++w) t += sred[w];
        s.E[rep] = -t / 2;
        s.bestE[rep] = kNoBest;
        s.accepts[rep] = 0ull;
    }
    __threadfence();
    G.sync();
}

// The last replica of an instance to finish its set-up: mega-iteration 0's tracking, then the
// first epoch, or the end when nothing is to run.
// `scratch`: the worker's shared memory, dead by now (the exchange stages a group in it).
__device__ void setup_done(const BatchDev &B, int k, unsigned char *scratch) {
    SolveDev s;
    load_desc(s, B.inst + k);
    const int replicas = s.T * s.R;
    const unsigned prev = atomicAdd(B.finish_inst + k, 1u);
    if (prev != (unsigned)replicas - 1u) return;
    __threadfence();
    B.finish_inst[k] = 0u;
    *s.start_ns = globaltimer_ns();
    for (int g = 0; g < s.T; ++g) track_exchange(s, g, 0, scratch);
    __threadfence();
    const int stop = *(volatile int32_t *)s.stop_epoch;
    if (0 < stop && 0 < __ldcg(B.max_megaiters + k)) {
        queue_push_instance(B, k, replicas);
    } else {
        publish_result(B, k);
        report_done(B, k);
        __threadfence();
        atomicSub(B.active, 1);
    }
}

// After replica-epoch `e` of instance k: the last replica to finish runs every group's
// tracking + exchange (lock step across groups, as one launch per epoch gives), then the next
// epoch or the end of the instance.
__device__ void epoch_done(const BatchDev &B, int k, int e, unsigned char *scratch) {
    SolveDev s;
    load_desc(s, B.inst + k);
    const int replicas = s.T * s.R;
    const unsigned prev = atomicAdd(B.finish_inst + k, 1u);
    if (prev != (unsigned)replicas - 1u) return;
    __threadfence();
    for (int g = 0; g < s.T; ++g) track_exchange(s, g, e + 1, scratch);
    B.finish_inst[k] = 0u;
    for (int g = 0; g < s.T; ++g) s.epoch[g] = e + 1;
    __threadfence();
    const int stop = *(volatile int32_t *)s.stop_epoch;
    if (e + 1 < stop && (int64_t)(e + 1) < __ldcg(B.max_megaiters + k)) {
        queue_push_instance(B, k, replicas);
    } else {
        __threadfence();
        if (B.serving) {
            publish_result(B, k);
            report_done(B, k);
        }
        atomicSub(B.active, 1);
    }
}

size_t batch_slice_bytes(int n, int bits) {
    const int isz = bits / 8, vec = 16 / isz;
    const int npad = (n + 3) & ~3;
    int lds = npad;
    if ((lds / vec) % 2 == 0) lds += vec;
    return align16(16 + std::max(SmemLayout(n, npad, lds, 1, isz).total, kExchangeScratchBytes));
}

template <class IT>
__global__ void __launch_bounds__(256) batch_kernel(BatchDev B) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int w = threadIdx.x / B.worker_threads;
    const int wt = threadIdx.x - w * B.worker_threads;
    const Grp G{wt, B.worker_threads, wt & 31, wt >> 5, B.worker_threads >> 5, 1 + w};
    unsigned char *slice = smem + (size_t)w * B.slice_bytes;
    volatile unsigned long long *hdr = reinterpret_cast<unsigned long long *>(slice);
    unsigned char *work = slice + 16;
    unsigned long long ticket = kNoTicket;   // held by G.tid == 0
    if (blockIdx.x == 0 && threadIdx.x == 0) *B.start_ns = globaltimer_ns();
    if (B.serving && threadIdx.x == 0) {   // tell the host this CTA is resident
        B.link.resident[blockIdx.x] = 1;
        __threadfence_system();
    }
    for (;;) {
        if (G.tid == 0) *hdr = queue_next(B, ticket);
        G.sync();
        const unsigned long long item = *hdr;
        G.sync();
        if (item == kDoneItem) break;
        if (item & kAdmitItem) {
            serve_admit(B, item, G);
            continue;
        }
        const int k = (int)(item >> 32);
        const int rep = (int)(item & 0x7fffffffull);
        SolveDev s;
        load_desc(s, B.inst + k);
        if (item & kSetupItem) {
            replica_setup<IT>(s, rep, G, reinterpret_cast<int32_t *>(work),
                              reinterpret_cast<long long *>(work + align16(4 * (size_t)s.n)));
            if (G.tid == 0) setup_done(B, k, work);
            continue;
        }
        const int e = *((volatile int32_t *)s.epoch);
        if (__ldcg(B.sym + k)) replica_epoch<IT, 1, true>(s, rep, 0, e, G, work);
        else replica_epoch<IT, 1, false>(s, rep, 0, e, G, work);
        G.sync();
        if (G.tid == 0) epoch_done(B, k, e, work);
    }
}

// Batch kernel for replicas that span a cluster of CL CTAs: rank 0 pops an item and writes it
// into every rank's header; the whole cluster runs the replica's epoch, rank 0 reports it.
template <class IT, int CL>
__global__ void __launch_bounds__(256, 1) batch_cluster_kernel(BatchDev B) {
    extern __shared__ __align__(16) unsigned char smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    unsigned long long *hdr = reinterpret_cast<unsigned long long *>(smem);
    unsigned char *work = smem + 16;
    const Grp G{(int)threadIdx.x, (int)blockDim.x, (int)(threadIdx.x & 31), (int)(threadIdx.x >> 5),
                (int)(blockDim.x >> 5), 0};
    unsigned long long ticket = kNoTicket;   // held by rank 0, thread 0
    if (blockIdx.x == 0 && threadIdx.x == 0) *B.start_ns = globaltimer_ns();
    if (B.serving && threadIdx.x == 0) {   // tell the host this CTA is resident
        B.link.resident[blockIdx.x] = 1;
        __threadfence_system();
    }
    cluster_barrier<CL>();
    for (;;) {
        if (rank == 0 && threadIdx.x == 0) {
            const unsigned long long item = queue_next(B, ticket);
#pragma unroll
            for (int r = 0; r < CL; ++r) *cluster.map_shared_rank(hdr, r) = item;
        }
        cluster_barrier<CL>();
        const unsigned long long item = *(volatile unsigned long long *)hdr;
        if (item == kDoneItem) break;
        if (item & kAdmitItem) {
            if (rank == 0) serve_admit(B, item, G);
        } else if (item & kSetupItem) {
            const int k = (int)(item >> 32);
            if (rank == 0) {
                SolveDev s;
                load_desc(s, B.inst + k);
                replica_setup<IT>(s, (int)(item & 0x7fffffffull), G, reinterpret_cast<int32_t *>(work),
                                  reinterpret_cast<long long *>(work + align16(4 * (size_t)s.n)));
                if (threadIdx.x == 0) setup_done(B, k, work);
            }
        } else {
            const int k = (int)(item >> 32), rep = (int)(item & 0x7fffffffull);
            SolveDev s;
            load_desc(s, B.inst + k);
            const int e = *((volatile int32_t *)s.epoch);
            bool ok;
            if (__ldcg(B.sym + k)) ok = replica_epoch<IT, CL, true>(s, rep, rank, e, G, work);
            else ok = replica_epoch<IT, CL, false>(s, rep, rank, e, G, work);
            // every rank has stored its rows of the force matrix (and fenced them) before rank 0
            // reports the epoch: the next epoch, or, once the instance ends, the next request
            // in its slot and memory, must not meet a late store
            cluster_barrier<CL>();
            if (!ok) {
                if (threadIdx.x == 0) set_error(B, kErrTimeout);
            } else if (rank == 0 && threadIdx.x == 0) {
                epoch_done(B, k, e, work);
            }
        }
        // the header is rewritten only after every rank has read it; this barrier also orders
        // the next pop after rank 0's report
        cluster_barrier<CL>();
    }
    cluster_barrier<CL>();
}

// Per-instance results of a batch, gathered on the device so the host reads them at once.
__global__ void batch_collect_kernel(const SolveDev *inst, int count, BatchResultDev *out,
                                     int32_t *perms, const long long *perm_off, long long *energies,
                                     const long long *energy_off) {
    const int k = blockIdx.x;
    if (k >= count) return;
    const SolveDev &s = inst[k];
    const int reps = s.T * s.R;
    __shared__ long long sb[128], sa[128];
    __shared__ unsigned long long sc[128];
    long long best = 0x7fffffffffffffffll, arg = 0;
    unsigned long long acc = 0;
    for (int r = threadIdx.x; r < reps; r += blockDim.x) {
        const long long v = __ldcg((const long long *)s.bestE + r);
        if (v < best) { best = v; arg = r; }
        acc += __ldcg(s.accepts + r);
    }
    sb[threadIdx.x] = best; sa[threadIdx.x] = arg; sc[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long b = sb[0], a = sa[0];
        unsigned long long c = sc[0];
        for (int t = 1; t < (int)blockDim.x; ++t) {
            if (sb[t] < b || (sb[t] == b && sa[t] < a)) { b = sb[t]; a = sa[t]; }
            c += sc[t];
        }
        BatchResultDev &o = out[k];
        o.best = b;
        o.arg = a;
        o.accepts = c;
        o.single_best = __ldcg((const long long *)s.single_best);
        o.target_epoch = __ldcg((const long long *)s.target_epoch);
        o.target_ns = __ldcg(s.target_ns);
        o.epoch = __ldcg(s.epoch);
        o.stop_epoch = __ldcg(s.stop_epoch);
        o.error = __ldcg(s.error);
        sa[0] = a;
    }
    __syncthreads();
    const long long a = sa[0];
    for (int q = threadIdx.x; q < s.n; q += blockDim.x)
        perms[perm_off[k] + q] = __ldcg(s.best_phi + a * s.n + q);
    for (int r = threadIdx.x; r < reps; r += blockDim.x)
        energies[energy_off[k] + r] = __ldcg((const long long *)s.E + r);
}

cudaError_t launch_collect(const SolveDev *inst, int count, BatchResultDev *out, int32_t *perms,
                           const long long *perm_off, long long *energies, const long long *energy_off,
                           cudaStream_t st) {
    if (count <= 0) return cudaSuccess;
    batch_collect_kernel<<<count, 128, 0, st>>>(inst, count, out, perms, perm_off, energies, energy_off);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ launchers

template <class IT, int CL, bool SYM> static void *epoch_fn(bool gp) {
    return gp ? reinterpret_cast<void *>(&epoch_kernel<IT, CL, SYM, true>)
              : reinterpret_cast<void *>(&epoch_kernel<IT, CL, SYM, false>);
}

// gp: the variant that records goal_print events (solver handles with goal_print set).
static void *epoch_kernel_ptr(int bits, int cl, bool sym, bool gp) {
#define PIMQAP_PICK(IT)                                                              \
    switch (cl) {                                                                    \
        case 1: return sym ? epoch_fn<IT, 1, true>(gp) : epoch_fn<IT, 1, false>(gp); \
        case 2: return sym ? epoch_fn<IT, 2, true>(gp) : epoch_fn<IT, 2, false>(gp); \
        case 4: return sym ? epoch_fn<IT, 4, true>(gp) : epoch_fn<IT, 4, false>(gp); \
        default: return nullptr;                                                     \
    }
    if (bits == 32) { PIMQAP_PICK(int32_t) }
    if (bits == 64) { PIMQAP_PICK(int64_t) }
#undef PIMQAP_PICK
    return nullptr;
}

template <class IT, int CL, bool SYM> static void *solve_fn(bool gp, int kind) {
    if (kind == 1) return reinterpret_cast<void *>(&solve_kernel<int32_t, CL, true, false, 1>);
    if (kind == 2)
        return gp ? reinterpret_cast<void *>(&solve_kernel<IT, CL, SYM, true, 2>)
                  : reinterpret_cast<void *>(&solve_kernel<IT, CL, SYM, false, 2>);
    return gp ? reinterpret_cast<void *>(&solve_kernel<IT, CL, SYM, true, 0>)
              : reinterpret_cast<void *>(&solve_kernel<IT, CL, SYM, false, 0>);
}

// The persistent solve kernel of a shape (kind: 0 generic, 1 binary-flow, 2 one-shot).
static void *solve_kernel_ptr(int bits, int cl, bool sym, bool gp, int kind) {
#define PIMQAP_PICK(IT)                                                                          \
    switch (cl) {                                                                                \
        case 1: return sym ? solve_fn<IT, 1, true>(gp, kind) : solve_fn<IT, 1, false>(gp, kind); \
        case 2: return sym ? solve_fn<IT, 2, true>(gp, kind) : solve_fn<IT, 2, false>(gp, kind); \
        case 4: return sym ? solve_fn<IT, 4, true>(gp, kind) : solve_fn<IT, 4, false>(gp, kind); \
        default: return nullptr;                                                                 \
    }
    if (kind == 1 && (bits != 32 || !sym)) return nullptr;
    if (bits == 32) { PIMQAP_PICK(int32_t) }
    if (bits == 64) { PIMQAP_PICK(int64_t) }
#undef PIMQAP_PICK
    return nullptr;
}

// The pipelined binary-flow epoch (2 x kPipeGroup threads).
static void *epoch_pipe_ptr(int cl) {
    switch (cl) {
        case 1: return reinterpret_cast<void *>(&epoch_kernel<int32_t, 1, true, false, 3>);
        case 2: return reinterpret_cast<void *>(&epoch_kernel<int32_t, 2, true, false, 3>);
        case 4: return reinterpret_cast<void *>(&epoch_kernel<int32_t, 4, true, false, 3>);
        default: return nullptr;
    }
}

// The paired binary-flow epoch (two replicas per CTA set).
static void *epoch_pair_ptr(int cl) {
    switch (cl) {
        case 1: return reinterpret_cast<void *>(&epoch_pair_kernel<1>);
        case 2: return reinterpret_cast<void *>(&epoch_pair_kernel<2>);
        case 4: return reinterpret_cast<void *>(&epoch_pair_kernel<4>);
        default: return nullptr;
    }
}

// The binary-flow epoch (int32 forces, symmetric instance, no goal_print events).
static void *epoch_bin_ptr(int cl) {
    switch (cl) {
        case 1: return reinterpret_cast<void *>(&epoch_kernel<int32_t, 1, true, false, 1>);
        case 2: return reinterpret_cast<void *>(&epoch_kernel<int32_t, 2, true, false, 1>);
        case 4: return reinterpret_cast<void *>(&epoch_kernel<int32_t, 4, true, false, 1>);
        default: return nullptr;
    }
}

template <class IT, int CL, bool SYM> static void *epoch_os_fn(bool gp) {
    return gp ? reinterpret_cast<void *>(&epoch_kernel<IT, CL, SYM, true, 2>)
              : reinterpret_cast<void *>(&epoch_kernel<IT, CL, SYM, false, 2>);
}

// The one-shot epoch.
static void *epoch_os_ptr(int bits, int cl, bool sym, bool gp) {
#define PIMQAP_PICK(IT)                                                                      \
    switch (cl) {                                                                            \
        case 1: return sym ? epoch_os_fn<IT, 1, true>(gp) : epoch_os_fn<IT, 1, false>(gp); \
        case 2: return sym ? epoch_os_fn<IT, 2, true>(gp) : epoch_os_fn<IT, 2, false>(gp); \
        case 4: return sym ? epoch_os_fn<IT, 4, true>(gp) : epoch_os_fn<IT, 4, false>(gp); \
        default: return nullptr;                                                             \
    }
    if (bits == 32) { PIMQAP_PICK(int32_t) }
    if (bits == 64) { PIMQAP_PICK(int64_t) }
#undef PIMQAP_PICK
    return nullptr;
}

static void *batch_fn(int bits, int cl) {
    if (bits == 32) {
        switch (cl) {
            case 1: return reinterpret_cast<void *>(&batch_kernel<int32_t>);
            case 2: return reinterpret_cast<void *>(&batch_cluster_kernel<int32_t, 2>);
            case 4: return reinterpret_cast<void *>(&batch_cluster_kernel<int32_t, 4>);
        }
    } else if (bits == 64) {
        switch (cl) {
            case 1: return reinterpret_cast<void *>(&batch_kernel<int64_t>);
            case 2: return reinterpret_cast<void *>(&batch_cluster_kernel<int64_t, 2>);
            case 4: return reinterpret_cast<void *>(&batch_cluster_kernel<int64_t, 4>);
        }
    }
    return nullptr;
}

cudaError_t launch_batch(const BatchDev &b, int bits, int cl, int grid, cudaStream_t st) {
    void *fn = batch_fn(bits, cl);
    if (!fn) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)(b.workers * b.worker_threads));
    cfg.dynamicSmemBytes = (size_t)b.workers * b.slice_bytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void *args[] = {const_cast<BatchDev *>(&b)};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

cudaError_t batch_occupancy(int bits, int cl, int threads, size_t smem, int *ctas_per_sm) {
    void *fn = batch_fn(bits, cl);
    if (!fn) return cudaErrorInvalidValue;
    if (cl == 1) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, fn, threads, smem);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)cl);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    cudaError_t e = cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg);
    *ctas_per_sm = clusters;   // for clusters: resident clusters on the whole device
    return e;
}

cudaError_t pair_occupancy(int cl, int threads, size_t smem, int *clusters) {
    void *fn = epoch_pair_ptr(cl);
    if (!fn) return cudaErrorInvalidValue;
    if (cl == 1) {
        int dev = 0, sms = 0, per = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, 2 * threads, smem);
        *clusters = per * sms;
        return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)cl);
    cfg.blockDim = dim3((unsigned)(2 * threads));
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaOccupancyMaxActiveClusters(clusters, fn, &cfg);
}

cudaError_t prepare_kernels() {
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    int maxsm = 0;
    err = cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (err != cudaSuccess) return err;
    for (int bits : {32, 64})
        for (int cl : {1, 2, 4})
            for (int sym = 0; sym < 2; ++sym)
                for (int gp = 0; gp < 2; ++gp) {
                    err = cudaFuncSetAttribute(epoch_kernel_ptr(bits, cl, sym != 0, gp != 0),
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
                    if (err != cudaSuccess) return err;
                    err = cudaFuncSetAttribute(epoch_os_ptr(bits, cl, sym != 0, gp != 0),
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
                    if (err != cudaSuccess) return err;
                }
    for (int bits : {32, 64})
        for (int cl : {1, 2, 4}) {
            err = cudaFuncSetAttribute(batch_fn(bits, cl), cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
            if (err != cudaSuccess) return err;
        }
    for (int bits : {32, 64})
        for (int cl : {1, 2, 4})
            for (int sym = 0; sym < 2; ++sym)
                for (int gp = 0; gp < 2; ++gp)
                    for (int kind = 0; kind < 3; ++kind) {
                        void *fn = solve_kernel_ptr(bits, cl, sym != 0, gp != 0, kind);
                        if (!fn) continue;
                        err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
                        if (err != cudaSuccess) return err;
                    }
    for (int cl : {1, 2, 4}) {
        err = cudaFuncSetAttribute(epoch_bin_ptr(cl), cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
        if (err != cudaSuccess) return err;
        err = cudaFuncSetAttribute(epoch_pair_ptr(cl), cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
        if (err != cudaSuccess) return err;
        err = cudaFuncSetAttribute(epoch_pipe_ptr(cl), cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
        if (err != cudaSuccess) return err;
    }
    return cudaSuccess;
}

cudaError_t launch_setup(const SolveDev &s, int bits, cudaStream_t st) {
    const dim3 tile(16, 16);
    const dim3 grid(s.T * s.R, (s.ldg + 15) / 16, (s.n + 15) / 16);
    if (bits == 32) {
        init_force_kernel<int32_t><<<grid, tile, 0, st>>>(s);
        init_energy_kernel<int32_t><<<s.T * s.R, 256, 0, st>>>(s);
    } else {
        init_force_kernel<int64_t><<<grid, tile, 0, st>>>(s);
        init_energy_kernel<int64_t><<<s.T * s.R, 256, 0, st>>>(s);
    }
    init_exchange_kernel<<<(s.T + 127) / 128, 128, 0, st>>>(s);
    return cudaGetLastError();
}

// The kernel the persistent solve runs for a solve's shape (the kind launch_epoch picks).
static void *solve_ptr_for(const SolveDev &s, int bits, int cluster, bool sym, bool bin) {
    const bool gp = s.ev.log != nullptr && s.ev.goal_print != 0;
    const int kind = s.os_chunk > 0 ? 2 : ((bin && bits == 32 && sym && (!gp || s.act > 0)) ? 1 : 0);
    return solve_kernel_ptr(bits, cluster, sym, gp, kind);
}

static cudaLaunchConfig_t solve_config(const SolveDev &s, int cluster, int threads, size_t smem,
                                       cudaStream_t st, cudaLaunchAttribute *attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(s.T * s.R * cluster));
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

cudaError_t solve_fits(const SolveDev &s, int bits, int cluster, bool sym, bool bin, int threads,
                       size_t smem, bool *fits) {
    *fits = false;
    void *fn = solve_ptr_for(s, bits, cluster, sym, bin);
    if (!fn) return cudaSuccess;
    smem = std::max(smem, exchange_scratch_bytes());
    const long long ctas = (long long)s.T * s.R * cluster;
    if (cluster == 1) {
        int dev = 0, sms = 0, per = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem);
        if (e != cudaSuccess) return e;
        *fits = (long long)per * sms >= ctas;
        return cudaSuccess;
    }
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = solve_config(s, cluster, threads, smem, nullptr, attr);
    cfg.gridDim = dim3((unsigned)cluster);
    int clusters = 0;
    cudaError_t e = cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg);
    if (e != cudaSuccess) return e;
    *fits = (long long)clusters * cluster >= ctas;
    return cudaSuccess;
}

cudaError_t launch_solve(const SolveDev &s, int bits, int cluster, bool sym, bool bin, int threads,
                         size_t smem, cudaStream_t st) {
    void *fn = solve_ptr_for(s, bits, cluster, sym, bin);
    if (!fn) return cudaErrorInvalidValue;
    smem = std::max(smem, exchange_scratch_bytes());
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = solve_config(s, cluster, threads, smem, st, attr);
    void *args[] = {const_cast<SolveDev *>(&s)};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

cudaError_t launch_epoch(const SolveDev &s, int bits, int cluster, bool sym, bool bin, int threads,
                         size_t smem, cudaStream_t st, bool pair, bool pipe) {
    const bool gp = s.ev.log != nullptr && s.ev.goal_print != 0;
    const bool binary = bin && bits == 32 && sym && (!gp || s.act > 0);
    pair = pair && binary;
    pipe = pipe && binary && !pair && s.act == 0;
    // clique-flow solves (s.act > 0) exist only in the binary-flow kernels
    void *fn = s.os_chunk > 0 ? epoch_os_ptr(bits, cluster, sym, gp)
               : pair         ? epoch_pair_ptr(cluster)
               : pipe         ? epoch_pipe_ptr(cluster)
               : binary       ? epoch_bin_ptr(cluster)
                              : epoch_kernel_ptr(bits, cluster, sym, gp);
    if (!fn) return cudaErrorInvalidValue;
    const int reps = s.T * s.R;
    if (!pair) smem = std::max(smem, exchange_scratch_bytes());   // the pair's sections hold it
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((pair ? (reps + 1) / 2 : reps) * cluster));
    cfg.blockDim = dim3((unsigned)(pair ? 2 * threads : (pipe ? 2 * kPipeGroup : threads)));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void *args[] = {const_cast<SolveDev *>(&s)};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

}  // namespace pimqap
