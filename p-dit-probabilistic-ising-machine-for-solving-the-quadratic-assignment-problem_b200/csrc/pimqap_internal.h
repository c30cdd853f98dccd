// pimqap_internal.h - device-side layout of a solve, shared by the kernels and the host
// runtime.  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace pimqap {

constexpr int kMaxN = 256;
constexpr int kMaxWarps = 8;           // kernels run with 64, 128 or 256 threads
constexpr int kMaxWarpsOs = 16;        // the one-shot epoch runs with up to 512
constexpr int32_t kNoStop = 0x7fffffff;
constexpr int64_t kNoBest = 2147483647;  // the reference's INT_MAX sentinel

// Device-side error word bits (SolveDev::error).
enum : int32_t {
    kErrBadPerm = 1,      // a permutation loaded from global memory is not a bijection
    kErrShape = 2,        // launch shape does not match the solve
    kErrTimeout = 4,      // a bounded wait for a peer CTA's data or a queue item gave up
    kErrHostLost = 8,     // serving: the host's heartbeat stopped
    kErrLaunchEnded = 16, // serving: a resident launch ended while serving (host-detected)
};

// One progress event, appended by the device for the reference's log lines.
//   kind_slot == -1: the tracking step of mega-iteration `megaiter` found replica `replica`
//                    of group `group` below the group's best (CPU_PIM.cpp:297-314); one event
//                    per lowering, in replica order, as the reference prints them.
//   kind_slot >= -2: a sweep of mega-iteration `megaiter` lowered the replica's best below
//                    goal_print (CPU_PIM.cpp:271-282); >= 0 is the slot of its permutation
//                    in EventLink::perm, -2 means the permutation store was full.
struct EventDev {
    int32_t megaiter, group, replica, kind_slot;
    int64_t energy;
    unsigned long long ns;     // %globaltimer
    int32_t tag, pad;          // batch member index (0 for a single solve)
};

// Where a solve appends its events (log == nullptr: no events).  Several solves of a batch
// may share one log and tell their events apart by tag.
struct EventLink {
    EventDev *log;
    int32_t *perm;             // [pcap][n] permutations of goal_print events
    unsigned int *count;       // [2] events appended, permutation slots taken (may pass caps)
    unsigned int cap, pcap;
    int64_t goal_print;        // 0: no goal_print events
    int32_t tag, pad;
};

// Everything one solve (one instance, T groups x R replicas) keeps in device memory.
// Arrays are indexed by replica slot rep = t * R + l or by group t.
struct SolveDev {
    int n, R, T, cap, spe;     // size, replicas/group, groups, rank slots, sweeps per epoch
    int ldg;                   // row stride of I in global memory (elements, 16-byte rows)
    int lds;                   // row stride of I in shared memory (elements)
    int ldm;                   // row stride of D, DT, F, FT (int32 elements, multiple of 4)
    int rpc;                   // rows of I per CTA (ceil(n / cluster size) rounded up to 4)
    int64_t goal;
    uint64_t seed;
    const int32_t *D, *DT, *F, *FT;  // n rows of ldm each, zero padded (DT = D transposed)
    const int32_t *Ddiag, *Fdiag;    // n each
    void *I;                   // [T*R][n][ldg] of int32 or int64
    int32_t *phi;              // [T*R][n]  facility at location
    int32_t *best_phi;         // [T*R][n]  phi of the replica's best state
    int64_t *E, *bestE;        // [T*R]
    double *beta;              // [T*R]     by replica slot, swapped by the exchange
    unsigned long long *accepts;   // [T*R]
    int32_t *order;            // [T][cap]  indexOfBetaOrder
    int32_t *tss;              // [T]       timeSinceSwap
    int64_t *group_best;       // [T]       threadBestE
    unsigned int *finish;      // [T]       replicas of the group done with this epoch
    int32_t *epoch;            // [T]       mega-iterations completed by the group
    int64_t *single_best;      // [1]       best over all groups (at tracking points)
    int32_t *stop_epoch;       // [1]       first epoch that must not run (goal reached)
    int64_t *target_epoch;     // [1]       mega-iteration whose tracking reached the goal
    unsigned long long *target_ns;  // [1]  %globaltimer at that tracking
    unsigned long long *start_ns;   // [1]  %globaltimer when sweeping started
    int32_t *error;            // [1]       kErr* bits
    EventLink ev;              // progress events (optional)
    int32_t act;               // > 0: clique-flow moves with facilities 0..act-1 active
    int32_t os_chunk;          // > 0: the one-shot update rule, force update in chunks of this
                               //      many swaps (0: sequential sweeps)
    int32_t os_xcol;           // one-shot with a cluster: peers push the force-matrix columns
                               //      the proposals need (0: the proposals read them remotely)
    int32_t os_mma;            // one-shot: the force update on the integer CUDA cores (0), on the
                               //      tensor cores by mma.sync (1) or by tcgen05 with the sums in
                               //      tensor memory (2); 1 and 2 only where exact for this
                               //      instance (small factors, sums below 2^24)
    int32_t bin_tc;            // binary-flow epoch: the 16-swap rewrite of the rows on the tcgen05
                               //      tensor cores (exact for this instance: small distance range)
    int32_t os_own_exp2;       // one-shot: the weights by this library's own 2^x (exp2f_neg: the
                               //      oracle's function) instead of CUDA's exp2f (the reference's)
    const double *replay_r;    // [sweeps][n] the uniform r of every update, given by the caller
                               //      (pimqap_sweep_replay); nullptr: drawn from the Philox stream
    // The persistent solve (one launch runs many mega-iterations; solve_kernel):
    int32_t *epoch_all;        // [1] mega-iterations every group has completed (the release word)
    unsigned int *finish_all;  // [1] groups done with the current mega-iteration
    const int32_t *run_end;    // [1] the launch stops before this mega-iteration
    const volatile int32_t *kill;  // [1] mapped host word: nonzero stops the launch at the next
                                   //     mega-iteration boundary (the host's timeout); may be null
};

// Compact per-instance result of a batch.
struct BatchResultDev {
    long long best, arg;
    unsigned long long accepts;
    long long single_best, target_epoch;
    unsigned long long target_ns;
    int32_t epoch, stop_epoch, error, pad;
};

// A served request as the host describes it (mapped memory); the device copies it in.
struct ServeDesc {
    SolveDev dev;                  // pointers into the device arena
    long long max_megaiters;
    unsigned long long head_bytes, tail_bytes;
    int32_t sym, bits;
};

// Host <-> running-kernel link of a serving launch.  Everything the host writes or reads lives
// in mapped pinned host memory, so the host serves without a single CUDA call (its streams
// could queue behind the resident launches); the claim counters live in device memory.
struct ServeLink {
    volatile unsigned long long *inbox;       // [inbox_mask+1] (slot << 32) | staging buffer
    volatile unsigned long long *inbox_tail;  // [1] entries the host has published
    unsigned long long *inbox_head;           // [1] entries the device has claimed (device memory)
    unsigned int inbox_mask;
    const volatile ServeDesc *desc;           // [slots]
    const unsigned char *staging;             // staging buffers of head images, `staging_stride` apart
    unsigned long long staging_stride;
    volatile int32_t *staging_busy;           // [buffers] the device clears it once copied
    volatile BatchResultDev *results;         // [slots]
    volatile int32_t *result_perm;            // [slots][256]
    volatile long long *result_energy;        // [slots][energy_stride]
    int energy_stride;
    volatile unsigned long long *done;        // [done_mask+1] slot of each finished instance
    volatile unsigned long long *done_seq;    // [done_mask+1] ring index + 1 once `done` is written
    unsigned long long *done_tail;            // [1] device counter (device memory)
    unsigned int done_mask;
    volatile unsigned long long *heartbeat;   // [1] the host increments it while it serves
    unsigned long long heartbeat_limit_ns;    // idle workers exit when it stalls this long
    volatile int32_t *error_host;             // [1] copy of the error word for the host
    volatile int32_t *resident;               // [grid] each CTA sets its entry when it starts
    SolveDev *inst_rw;                        // writable view of the device descriptor table
    int32_t *sym_rw;
    int64_t *maxm_rw;
};

// Item flag of a serving launch: replica set-up (force matrix, energy) instead of an epoch.
constexpr unsigned int kSetupItem = 0x80000000u;

// A batch of independent solves run by one persistent launch.  Work items are replica-epochs
// (instance k, replica rep) in a ring buffer; the last replica of an instance to finish an
// epoch runs the tracking / exchange of all its groups and enqueues the next epoch.
struct BatchDev {
    const SolveDev *inst;            // [count] per-instance descriptors
    const int32_t *sym;              // [count] 1 when D and F are symmetric
    const int64_t *max_megaiters;    // [count]
    unsigned int *finish_inst;       // [count] replicas done with the current epoch
    int count;
    unsigned long long *q_items;     // [qmask + 1] (instance << 32) | replica
    unsigned long long *q_seq;       // [qmask + 1] ticket + 1 once the slot holds that ticket
    unsigned long long *q_head;      // [1] next ticket to pop
    unsigned long long *q_tail;      // [1] next ticket to push
    unsigned int qmask;
    int32_t *active;                 // [1] instances still running
    volatile int32_t *shutdown;      // [1] nonzero: workers exit once no instance is active
    int32_t *error;                  // [1] kErr* bits
    unsigned long long *start_ns;    // [1] %globaltimer when the launch began
    int serving;                     // nonzero: `link` is live (instances arrive while running)
    ServeLink link;
    int worker_threads;              // threads of one replica worker (a multiple of 32)
    int workers;                     // workers per CTA (<= 8)
    unsigned int slice_bytes;        // shared memory of one worker
};

// Shared memory of one replica worker of the batch kernel (single-CTA replica of size n).
size_t batch_slice_bytes(int n, int bits);

// The persistent batch launch: grid CTAs (clusters of cl) of workers * worker_threads threads.
cudaError_t launch_batch(const BatchDev &b, int bits, int cl, int grid, cudaStream_t st);

// Residency of the batch kernel for this shape: CTAs per SM for cl == 1, else resident
// clusters on the device.
cudaError_t batch_occupancy(int bits, int cl, int threads, size_t smem, int *out);

// Gathers every instance's result, best permutation (perms + perm_off[k], n entries) and
// final replica energies (energies + energy_off[k], T*R entries).
cudaError_t launch_collect(const SolveDev *inst, int count, BatchResultDev *out, int32_t *perms,
                           const long long *perm_off, long long *energies, const long long *energy_off,
                           cudaStream_t st);

// Records msg as the calling thread's pimqap_last_error() text.
void set_last_error(const char *msg);

// Shared memory the tracking / exchange step needs once an epoch is over (the sweep kernels are
// launched with at least this much).
size_t exchange_scratch_bytes();

// Shared memory of one CTA of the epoch kernel.
size_t epoch_smem_bytes(int n, int rpc, int lds, int cluster, int bits);
// Shared memory of the binary-flow epoch kernel (0 / 1 flows and int16 distances resident).
size_t epoch_smem_bytes_bin(int n, int rpc, int lds, int cluster, bool tc_rewrite);
// Shared memory of the paired binary-flow epoch kernel (two replicas per CTA set).
size_t epoch_smem_bytes_bin_pair(int n, int rpc, int lds, int cluster);
// Shared memory of the one-shot epoch kernel (force update in chunks of `chunk` swaps; mma:
// 0 integer CUDA cores, 1 mma.sync, 2 tcgen05, as SolveDev::os_mma).
size_t epoch_smem_bytes_os(int n, int rpc, int lds, int cluster, int bits, int chunk, bool sym, bool xcol,
                           int mma);
// Tensor-memory columns one CTA of the tcgen05 one-shot epoch holds for its whole life.
int os_tmem_columns(int n);

// Resident clusters (CTAs for cl == 1) of the paired binary-flow epoch on the whole device.
cudaError_t pair_occupancy(int cl, int threads, size_t smem, int *clusters);

// The persistent solve: every replica (CTA or cluster) resident for the whole launch, which runs
// mega-iterations from *epoch_all up to *run_end (or the goal / kill stop) with a bounded
// device-side barrier between them.  Returns cudaErrorInvalidValue for shapes it lacks.
cudaError_t launch_solve(const SolveDev &s, int bits, int cluster, bool sym, bool bin, int threads,
                         size_t smem, cudaStream_t st);
// Whether every replica of the solve can be resident at once for launch_solve's kernel.
cudaError_t solve_fits(const SolveDev &s, int bits, int cluster, bool sym, bool bin, int threads,
                       size_t smem, bool *fits);

// One-time kernel attributes (dynamic shared memory, non-portable cluster size).
cudaError_t prepare_kernels();

// setup(): force matrices + energies of every replica from its phi, then the tracking /
// exchange step of mega-iteration 0 (which also records start_ns).
cudaError_t launch_setup(const SolveDev &s, int bits, cudaStream_t st);

// One epoch: spe sweeps of every replica, then each group's tracking + exchange.  pair: the
// binary-flow kernel with two replicas per CTA set (threads per replica; smem of the pair).
cudaError_t launch_epoch(const SolveDev &s, int bits, int cluster, bool sym, bool bin, int threads,
                         size_t smem, cudaStream_t st, bool pair = false, bool pipe = false);
// Shared memory of the pipelined binary-flow epoch (deltas of the next update computed while
// the current one picks; 256 threads).
size_t epoch_smem_bytes_pipe(int n, int rpc, int lds);

}  // namespace pimqap
