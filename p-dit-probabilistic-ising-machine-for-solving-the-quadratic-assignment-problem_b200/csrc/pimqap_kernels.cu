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
#include <cuda_runtime.h>

#include <cstdint>

#include "pimqap_internal.h"

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

// Offsets (bytes) of the epoch kernel's shared-memory sections.
struct SmemLayout {
    size_t I, phi, inv, bphi, Dd, Fd, dE, u1, u2, v1, v2, wmax, wsum, r, misc, total;
    __host__ __device__ SmemLayout(int n, int rpc, int lds, int cluster, int isz) {
        const size_t npad = (size_t)((n + 3) & ~3);
        const size_t rpad = (size_t)((rpc + 3) & ~3);
        size_t o = 0;
        I = o;    o = align16(o + (size_t)rpc * lds * isz);
        phi = o;  o = align16(o + npad * 4);
        inv = o;  o = align16(o + npad * 4);
        bphi = o; o = align16(o + npad * 4);
        Dd = o;   o = align16(o + npad * 4);
        Fd = o;   o = align16(o + npad * 4);
        dE = o;   o = align16(o + 2 * npad * isz);
        u1 = o;   o = align16(o + rpad * isz);
        u2 = o;   o = align16(o + rpad * isz);
        v1 = o;   o = align16(o + npad * isz);
        v2 = o;   o = align16(o + npad * isz);
        wmax = o; o = align16(o + 2 * (size_t)cluster * kMaxWarps * isz);
        wsum = o; o = align16(o + kMaxWarps * sizeof(double));
        r = o;    o = align16(o + 2 * sizeof(double));
        misc = o; o = align16(o + 4 * sizeof(int));
        total = o;
    }
};

size_t epoch_smem_bytes(int n, int rpc, int lds, int cluster, int bits) {
    return SmemLayout(n, rpc, lds, cluster, bits / 8).total;
}

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

// ------------------------------------------------------------------ tracking + exchange

// Best tracking, replica exchange and goal test of group g at the start of mega-iteration
// e_next (CPU_PIM.cpp:295-348).  Runs on one thread after every replica of the group has
// finished its sweeps; reads their energies through L2.
__device__ void track_exchange(const SolveDev &s, int g, int e_next) {
    const int R = s.R, cap = s.cap;
    volatile int64_t *E = s.E + (size_t)g * R;
    volatile int64_t *bestE = s.bestE + (size_t)g * R;
    volatile double *beta = s.beta + (size_t)g * R;
    volatile int32_t *order = s.order + (size_t)g * cap;
    int tss = s.tss[g] + 1;                                  // :295
    int64_t gb = s.group_best[g];
    bool found = false;
    for (int l = 0; l < R; ++l) {                            // :297-314
        const int64_t b = bestE[l];
        if (b < gb) {
            found = true;
            gb = b;
            tss = 0;
        }
    }
    if (found) atomicMin((long long *)s.single_best, (long long)gb);
    for (int l = 0; l < R - 1; ++l) {                        // :324-337
        const int i1 = order[l], i2 = order[l + 1];
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
    if (tss > 100) {                                         // :339-344, slot cap-1
        const int i1 = order[cap - 1], i2 = order[0];
        order[cap - 1] = i2;
        order[0] = i1;
        const double tb = beta[i1];
        beta[i1] = beta[i2];
        beta[i2] = tb;
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
        sD[ty][tx] = (i < n && jok) ? s.D[i * n + j] : 0;
        sDT[ty][tx] = (i < n && jok) ? s.DT[i * n + j] : 0;
        sFp[ty][tx] = (arow < n && jok) ? s.F[arow * n + pj] : 0;
        sFTp[ty][tx] = (arow < n && jok) ? s.FT[arow * n + pj] : 0;
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

template <class IT, int CL, bool SYM>
__global__ void __launch_bounds__(256) epoch_kernel(SolveDev s) {
    using U = typename Unsigned<IT>::type;
    constexpr int VEC = Vec<IT>::kN;
    extern __shared__ __align__(16) unsigned char smem[];

    const int n = s.n;
    const int tid = threadIdx.x, BT = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = BT >> 5;
    int rank = 0;
    if constexpr (CL > 1) rank = (int)cg::this_cluster().block_rank();
    const int rep = blockIdx.x / CL;
    const int g = rep / s.R, l = rep - g * s.R;

    // Every CTA of a group reads the same epoch and stop values: stop_epoch only drops to
    // epoch+1 during this launch, so the test below cannot differ inside a cluster or group.
    const int e = *((volatile int32_t *)s.epoch + g);
    if (e >= *(volatile int32_t *)s.stop_epoch) return;

    const int rpc = s.rpc, lds = s.lds;
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
    IT *s_dE = reinterpret_cast<IT *>(smem + L.dE);
    IT *s_u1 = reinterpret_cast<IT *>(smem + L.u1);
    IT *s_u2 = reinterpret_cast<IT *>(smem + L.u2);
    IT *s_v1 = reinterpret_cast<IT *>(smem + L.v1);
    IT *s_v2 = reinterpret_cast<IT *>(smem + L.v2);
    IT *s_wmax = reinterpret_cast<IT *>(smem + L.wmax);
    double *s_wsum = reinterpret_cast<double *>(smem + L.wsum);
    double *s_r = reinterpret_cast<double *>(smem + L.r);
    int *s_misc = reinterpret_cast<int *>(smem + L.misc);   // [0] pick, [1] improved-at

    // ---- load the replica
    {
        const IT *gI = reinterpret_cast<const IT *>(s.I) + ((size_t)rep * n + row0) * s.ldg;
        const int nvg = s.ldg / VEC;
        for (int idx = tid; idx < rows * nvg; idx += BT) {
            const int k = idx / nvg, v = idx - k * nvg;
            *reinterpret_cast<Vec<IT> *>(sI + (size_t)k * lds + v * VEC) =
                *reinterpret_cast<const Vec<IT> *>(gI + (size_t)k * s.ldg + v * VEC);
        }
        const int32_t *gphi = s.phi + (size_t)rep * n;
        for (int q = tid; q < npad; q += BT) {
            // an entry outside [0, n) would index out of range: clamp it and flag the error
            int p = q < n ? gphi[q] : 0;
            if ((unsigned)p >= (unsigned)n) {
                atomicOr(s.error, kErrBadPerm);
                p = 0;
            }
            s_phi[q] = p;
            s_bphi[q] = p;
            s_inv[q] = 0;
            s_Dd[q] = q < n ? s.Ddiag[q] : 0;
            s_Fd[q] = q < n ? s.Fdiag[q] : 0;
        }
        if (tid == 0) {
            s_misc[0] = 0x7fffffff;
            s_misc[1] = -1;
        }
    }
    __syncthreads();
    for (int q = tid; q < n; q += BT) s_inv[s_phi[q]] = q;

    // Pointers into every CTA of the cluster (delta / maxima scatter, remote rows of I).
    IT *dE_at[CL];
    IT *wmax_at[CL];
    if constexpr (CL > 1) {
        cg::cluster_group cluster = cg::this_cluster();
#pragma unroll
        for (int r = 0; r < CL; ++r) {
            dE_at[r] = cluster.map_shared_rank(s_dE, r);
            wmax_at[r] = cluster.map_shared_rank(s_wmax, r);
        }
    } else {
        dE_at[0] = s_dE;
        wmax_at[0] = s_wmax;
    }
    cluster_barrier<CL>();   // every CTA of the cluster is resident and initialised

    const double beta = s.beta[rep];
    const double cut_span = 20.0 / beta;                    // CPU_PIM.cpp:234
    int64_t E = s.E[rep], bestE = s.bestE[rep];
    unsigned long long accepts = 0;
    const uint32_t k0 = (uint32_t)s.seed, k1 = (uint32_t)(s.seed >> 32);
    const int K = (n + BT - 1) / BT;                         // weights per thread (<= 4)
    const int nvec = npad / VEC;
    int upd = 0;                                             // update counter (buffer parity)

    for (int sw = 0; sw < s.spe; ++sw) {
        const uint32_t sweep = (uint32_t)(e * s.spe + sw);
        for (int i = 0; i < n; ++i, ++upd) {
            const int buf = upd & 1;
            IT *dEb = s_dE + buf * npad;
            if (tid == 0) {
                uint32_t w0, w1;
                philox_2words((uint32_t)i, sweep, (uint32_t)l, (uint32_t)g, k0, k1, w0, w1);
                s_r[buf] = canonical53(w0, w1);
            }
            const int a = s_phi[i];

            // ---- 1. swap deltas of the candidates this CTA owns
            IT lmax = 0;                                     // max starts at 0 (:208)
            {
                const int owner = i / rpc;
                const IT *Ii = sI + (size_t)(i - owner * rpc) * lds;
                if constexpr (CL > 1) {
                    if (owner != rank) Ii = cg::this_cluster().map_shared_rank(Ii, owner);
                }
                const IT Iia = Ii[a];
                const int32_t Dii = s_Dd[i], Faa = s_Fd[a];
                for (int jj = tid; jj < rows; jj += BT) {
                    const int j = row0 + jj;
                    const int b = s_phi[j];
                    const IT *Ij = sI + (size_t)jj * lds;
                    const U dd = (U)(IT)Dii + (U)(IT)s_Dd[j] - (U)(IT)__ldg(s.D + i * n + j) -
                                 (U)(IT)__ldg(s.DT + i * n + j);
                    const U ff = (U)(IT)Faa + (U)(IT)s_Fd[b] - (U)(IT)__ldg(s.F + a * n + b) -
                                 (U)(IT)__ldg(s.FT + a * n + b);
                    const IT dE = (IT)((U)Ii[b] + (U)Ij[a] - (U)Iia - (U)Ij[b] - dd * ff);
#pragma unroll
                    for (int r = 0; r < CL; ++r) dE_at[r][buf * npad + b] = dE;
                    lmax = dE > lmax ? dE : lmax;
                }
            }
            lmax = warp_max(lmax);
            if (lane == 0) {
#pragma unroll
                for (int r = 0; r < CL; ++r) wmax_at[r][(buf * CL + rank) * kMaxWarps + warp] = lmax;
            }
            cluster_barrier<CL>();                           // S1
            if (tid == 0) s_misc[0] = 0x7fffffff;

            // ---- 2. heat-bath weights, prefix sum in b order, threshold pick
            IT M = 0;
            for (int q = 0; q < CL * nwarps; ++q) {
                const int rr = q / nwarps, ww = q - rr * nwarps;
                const IT v = s_wmax[(buf * CL + rr) * kMaxWarps + ww];
                M = v > M ? v : M;
            }
            const long long cut = cutoff_trunc(__dsub_rn((double)M, cut_span));   // :234-235
            double p[4];
            double local = 0.0;
            const int b0 = tid * K;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                p[k] = local;
                if (k < K) {
                    const int b = b0 + k;
                    if (b < n) {
                        const IT d = dEb[b];
                        if ((long long)d > cut) local = __dadd_rn(local, exp2(__dmul_rn(beta, (double)d)));
                    }
                    p[k] = local;
                }
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
            __syncthreads();                                 // S2
            double base = 0.0, total = 0.0;
            for (int w = 0; w < nwarps; ++w) {
                if (w == warp) base = total;
                total = __dadd_rn(total, s_wsum[w]);
            }
            const double target = __dmul_rn(s_r[buf], total);   // :247
            const double X = __dadd_rn(base, excl);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (k < K && b0 + k < n) {
                    if (__dadd_rn(X, p[k]) >= target) {     // :251
                        atomicMin(&s_misc[0], b0 + k);
                        break;
                    }
                }
            }
            __syncthreads();                                 // S3
            const int bs = s_misc[0];
            if (bs >= n || bs == a) continue;                // no move / self move (:252)

            // ---- 3. accepted swap: i gets facility bs, j = phiinv(bs) gets a
            const int j = s_inv[bs];
            const IT dEsel = dEb[bs];
            for (int k = tid; k < rows; k += BT) {
                const int kk = row0 + k;
                if constexpr (SYM) {
                    s_u1[k] = (IT)(2 * ((U)(IT)__ldg(s.D + j * n + kk) - (U)(IT)__ldg(s.D + i * n + kk)));
                } else {
                    s_u1[k] = (IT)((U)(IT)__ldg(s.DT + j * n + kk) - (U)(IT)__ldg(s.DT + i * n + kk));
                    s_u2[k] = (IT)((U)(IT)__ldg(s.D + j * n + kk) - (U)(IT)__ldg(s.D + i * n + kk));
                }
            }
            for (int c = tid; c < npad; c += BT) {
                if constexpr (SYM) {
                    s_v1[c] = c < n ? (IT)((U)(IT)__ldg(s.F + bs * n + c) - (U)(IT)__ldg(s.F + a * n + c)) : (IT)0;
                } else {
                    s_v1[c] = c < n ? (IT)((U)(IT)__ldg(s.FT + bs * n + c) - (U)(IT)__ldg(s.FT + a * n + c)) : (IT)0;
                    s_v2[c] = c < n ? (IT)((U)(IT)__ldg(s.F + bs * n + c) - (U)(IT)__ldg(s.F + a * n + c)) : (IT)0;
                }
            }
            __syncthreads();                                 // S4
            if (tid == 0) {
                s_phi[i] = bs;                               // :257-261
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
            // I[k][c] += (D[k][j]-D[k][i])(F[c][b]-F[c][a]) + (D[j][k]-D[i][k])(F[b][c]-F[a][c])
            if (nvec <= BT) {
                const int kstep = BT / nvec;
                const int cv = tid % nvec;
                int k = tid / nvec;
                if (k < kstep) {
                    const Vec<IT> v1 = *reinterpret_cast<const Vec<IT> *>(s_v1 + cv * VEC);
                    Vec<IT> v2;
                    if constexpr (!SYM) v2 = *reinterpret_cast<const Vec<IT> *>(s_v2 + cv * VEC);
                    for (; k < rows; k += kstep) {
                        Vec<IT> *dst = reinterpret_cast<Vec<IT> *>(sI + (size_t)k * lds + cv * VEC);
                        Vec<IT> x = *dst;
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
                        *dst = x;
                    }
                }
            } else {
                for (int cv = tid; cv < nvec; cv += BT) {
                    const Vec<IT> v1 = *reinterpret_cast<const Vec<IT> *>(s_v1 + cv * VEC);
                    Vec<IT> v2;
                    if constexpr (!SYM) v2 = *reinterpret_cast<const Vec<IT> *>(s_v2 + cv * VEC);
                    for (int k = 0; k < rows; ++k) {
                        Vec<IT> *dst = reinterpret_cast<Vec<IT> *>(sI + (size_t)k * lds + cv * VEC);
                        Vec<IT> x = *dst;
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
                        *dst = x;
                    }
                }
            }
            cluster_barrier<CL>();                           // S5: new rows and phi visible
            if (s_misc[1] == upd) {
                for (int q = tid; q < n; q += BT) s_bphi[q] = s_phi[q];
            }
        }
    }

    // ---- store the replica, then the last replica of the group runs the exchange
    cluster_barrier<CL>();   // no CTA of the cluster reads this CTA's rows any more
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
            s.accepts[rep] += accepts;
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            const unsigned prev = atomicAdd(s.finish + g, 1u);
            if (prev == (unsigned)s.R - 1u) {
                __threadfence();
                track_exchange(s, g, e + 1);
                s.finish[g] = 0u;
                s.epoch[g] = e + 1;
                __threadfence();
            }
        }
    }
}

// ------------------------------------------------------------------ launchers

template <class IT, int CL, bool SYM> static void *epoch_fn() {
    return reinterpret_cast<void *>(&epoch_kernel<IT, CL, SYM>);
}

static void *epoch_kernel_ptr(int bits, int cl, bool sym) {
#define PIMQAP_PICK(IT)                                                        \
    switch (cl) {                                                              \
        case 1: return sym ? epoch_fn<IT, 1, true>() : epoch_fn<IT, 1, false>(); \
        case 2: return sym ? epoch_fn<IT, 2, true>() : epoch_fn<IT, 2, false>(); \
        case 4: return sym ? epoch_fn<IT, 4, true>() : epoch_fn<IT, 4, false>(); \
        default: return nullptr;                                               \
    }
    if (bits == 32) { PIMQAP_PICK(int32_t) }
    if (bits == 64) { PIMQAP_PICK(int64_t) }
#undef PIMQAP_PICK
    return nullptr;
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
            for (int sym = 0; sym < 2; ++sym) {
                err = cudaFuncSetAttribute(epoch_kernel_ptr(bits, cl, sym != 0),
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
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

cudaError_t launch_epoch(const SolveDev &s, int bits, int cluster, bool sym, int threads,
                         size_t smem, cudaStream_t st) {
    void *fn = epoch_kernel_ptr(bits, cluster, sym);
    if (!fn) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(s.T * s.R * cluster));
    cfg.blockDim = dim3((unsigned)threads);
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
