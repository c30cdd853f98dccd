// pimqap_plan.h - per-instance planning and staging shared by the solve, batch and serving
// paths of the host runtime.  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "pimqap.h"
#include "pimqap_internal.h"

#define PQ_CUDA(x)                                                                          \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess)                                                              \
            return ::pimqap::detail::fail(PIMQAP_ERR_CUDA,                                  \
                                          std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace pimqap {
namespace detail {

// Records msg as pimqap_last_error() of the calling thread and returns st.
pimqap_status fail(pimqap_status st, const std::string &msg);

// Phase timing on stderr when the environment variable PIMQAP_TRACE is set.
void trace(const char *phase);

int round_up(int x, int m);
inline size_t carve_size(size_t bytes) { return (bytes + 255) & ~size_t(255); }
template <class T> T *carve(char *&cur, size_t count) {
    T *p = reinterpret_cast<T *>(cur);
    cur += carve_size(count * sizeof(T));
    return p;
}

// Philox4x32-10 (Salmon et al., SC'11) on the host: the ten rounds applied to counter c in
// place, key (k0, k1).
inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
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

// The initial permutation of the next group (CPU_PIM.cpp:143-162): identity, then for each
// location i one draw j in [0, n) from the shared stream and the transposition (i j).
// Groups draw one after another from the same engine.
void shuffle_group(ShuffleEngine &eng, int n, int32_t *perm);

// Initial permutations of T groups (CPU_PIM.cpp:134-162) from the shuffle stream of `seed`.
std::vector<int32_t> initial_perms(int n, int T, uint64_t seed);

pimqap_status check_params(const pimqap_instance *inst, const pimqap_params *p);

// Everything decided for one instance before device memory is touched.  Device memory of an
// instance is a head (uploaded from the host) and a tail (state that starts at zero).
struct Plan {
    int n = 0, T = 0, R = 0, cap = 0, spe = 0;
    int bits = 32, cl = 1, threads = 256;
    int npad = 0, lds = 0, ldm = 0, rpc = 0;
    bool sym = false;
    bool bin = false;      // the solve path may run the binary-flow epoch kernel
    size_t smem = 0;       // epoch kernel shared memory per CTA (the generic kernel)
    size_t smem_bin = 0;   // the binary-flow kernel's (when bin; of the pair when pair)
    bool pair = false;     // the solve path runs two replicas per CTA set (binary-flow kernel)
    bool pipe = false;     // the solve path runs the pipelined binary-flow epoch
    int act = 0;           // clique-flow moves with facilities 0..act-1 active (0 = off)
    int os_chunk = 0;      // > 0: the one-shot rule (swaps per force-update chunk)
    int os_xcol = 0;       // one-shot: peers push the force-matrix columns of the proposals
    int os_mma = 0;        // one-shot: force update on CUDA cores (0), mma.sync (1), tcgen05 (2)
    int os_own_exp2 = 0;   // one-shot: weights by this library's 2^x (1) or CUDA's exp2f (0)
    bool bin_tc = false;   // binary-flow epoch: the row rewrite on the tcgen05 tensor cores
    size_t head = 0, tail = 0, total = 0;
    int64_t h2d_bytes = 0;
};

// Symmetry of D and F, and the force-matrix width a bound on |I| and the deltas allows
// (32, 64, or 0 when not even int64 is provably safe).
struct InstanceInfo {
    bool symmetric = false;
    int bits_needed = 32;
    bool binary_flow = false;   // every flow is 0 or 1
    bool dist16 = false;        // every distance fits in int16
    int clique = 0;             // A > 0: F[a][b] = 1 exactly for a != b < A, and diag(D) = 0
    int64_t dmin = 0, dmax = 0, fmin = 0, fmax = 0;   // value ranges of D and F
};
InstanceInfo analyse(int n, const int32_t *F, const int32_t *D);

// Makes `device` current, checks it is an sm_100 part and prepares the kernels.
pimqap_status open_device(int device, int *maxsm);

// Force-matrix width, symmetry, launch shape (threads; the smallest cluster whose row share
// of the force matrix fits one CTA, or want_cluster), strides and device footprint.
pimqap_status plan_instance(const pimqap_instance *inst, const pimqap_params *params, size_t maxsm,
                            int want_cluster, Plan *out, const InstanceInfo *known = nullptr);

// Solver path only: replaces *P by the paired binary-flow layout (two replicas per CTA set,
// on the smallest cluster of at least P->cl CTAs that holds it) when params->replica_pairing
// is 2; 0 and 1 keep one replica per CTA set.
pimqap_status plan_pairing(const pimqap_instance *inst, const pimqap_params *params, size_t maxsm,
                           Plan *P);

// Device pointers of one instance carved from its head and tail regions.
void carve_instance(const Plan &P, char *head, char *tail, SolveDev *out);

// Host image of the head region (P.head bytes), laid out as carve_instance lays it out.
void fill_head(const pimqap_instance *inst, const pimqap_params *params, const Plan &P,
               char *mirror);

// Head upload + tail clear + setup kernels for one instance in `base` (P.total bytes) on
// stream q.  The host image is kept in `keep` until the caller syncs q.  `ev` (may be null)
// is the event log the solve appends to.
pimqap_status stage_instance(const pimqap_instance *inst, const pimqap_params *params,
                             const Plan &P, char *base, SolveDev *out, cudaStream_t q,
                             std::vector<std::vector<char>> &keep, const EventLink *ev = nullptr);

}  // namespace detail
}  // namespace pimqap
