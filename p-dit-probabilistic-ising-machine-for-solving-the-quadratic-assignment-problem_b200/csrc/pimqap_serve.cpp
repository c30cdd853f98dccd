// pimqap_serve.cpp - continuous-batching solve service (no reference counterpart).
//
// One persistent launch per class of replica shape stays resident on its share of the SMs
// (the autotuner sizes classes and shares from a sample of the expected requests).  While they
// run, the server thread makes no CUDA call at all (a stream operation could queue behind a
// resident launch in a shared hardware queue and never run); host and device talk only
// through mapped pinned memory:
//   - admission: when a slot of the request's class and device memory (a first-fit arena in
//     the budget) are free, the thread writes the request's head image (matrices, initial
//     permutations, betas, rank slots) into a staging buffer and its descriptor into the
//     slot, then publishes (slot, buffer) in the class's inbox ring;
//   - an idle device worker claims the entry, copies descriptor and head into device memory,
//     clears the state, and queues one set-up item per replica (force matrix and energy on the
//     device), after which the replica-epochs run as in a batch;
//   - the last replica to finish writes the result, best permutation and final energies into
//     the slot's mapped result area and posts the slot on the completion ring;
//   - the thread increments each class's heartbeat, which bounds every idle device wait.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "pimqap.h"
#include "pimqap_batch.h"
#include "pimqap_internal.h"
#include "pimqap_plan.h"

using Clock = std::chrono::steady_clock;

namespace pimqap {
namespace detail {

// First-fit allocator over [0, size) with 256-byte granules and coalescing.
class Arena {
  public:
    void reset(size_t size) {
        free_.clear();
        free_[0] = size;
        size_ = size;
        used_ = 0;
    }
    bool alloc(size_t bytes, size_t *off) {
        bytes = carve_size(bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const size_t rest = it->second - bytes;
            const size_t at = it->first + bytes;
            free_.erase(it);
            if (rest) free_[at] = rest;
            used_ += bytes;
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        bytes = carve_size(bytes);
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t size() const { return size_; }
    size_t used() const { return used_; }

  private:
    std::map<size_t, size_t> free_;
    size_t size_ = 0, used_ = 0;
};

struct Request {
    int64_t ticket = 0;
    std::vector<int32_t> F, D;
    pimqap_instance inst{};
    pimqap_params params{};
    Plan plan;
    InstanceInfo info;
    int cls = -1, slot = -1;
    size_t off = 0;
    enum State { kPending, kRunning, kDone, kFailed } state = kPending;
    pimqap_status status = PIMQAP_OK;
    Clock::time_point t_submit, t_admit, t_done;
    SolveDev dev{};
    pimqap_result result{};
    std::vector<int32_t> perm;
    std::vector<int64_t> energies;
    int64_t maxm = 0;
    double work = 0;           // estimated cost, counted in its class's load until it completes
};

struct ServeClass {
    BatchClass shape;
    double load = 0;           // estimated cost of the requests routed here and not yet done
    int slots = 0;
    std::vector<int> free_slots;
    std::vector<int64_t> slot_ticket;
    size_t qcap = 0, replicas_in_flight = 0;
    char *dbase = nullptr;
    SolveDev *d_inst = nullptr;
    int32_t *d_sym = nullptr;
    int64_t *d_maxm = nullptr;
    char *hbase = nullptr;   // mapped pinned host block
    volatile unsigned long long *h_inbox = nullptr, *h_inbox_tail = nullptr;
    volatile unsigned long long *h_done = nullptr, *h_done_seq = nullptr, *h_heartbeat = nullptr;
    volatile int32_t *h_shutdown = nullptr, *h_error = nullptr, *h_resident = nullptr;
    volatile ServeDesc *h_desc = nullptr;
    volatile BatchResultDev *h_res = nullptr;
    volatile int32_t *h_perm = nullptr;
    volatile long long *h_energy = nullptr;
    unsigned inbox_cap = 0, done_cap = 0;
    unsigned long long inbox_tail = 0, done_head = 0;
    cudaStream_t stream = nullptr;
    BatchDev B{};
};

// Requests a served instance may hold at once: up to 1024 replicas (groups x replicas).
constexpr int kServeMaxReplicas = 1024;
constexpr int kServeMaxRankSlots = 65536;   // groups x rank slots of a served request
constexpr int kStagingBuffers = 8;
constexpr int kMaxResidentCtas = 1024;     // CTAs of one resident launch (at most one per SM)

struct Server {
    pimqap_server_config cfg{};
    int device = 0, sms = 0, maxsm = 0;
    std::vector<ServeClass> classes;
    Arena arena;
    char *arena_base = nullptr;
    char *staging = nullptr;              // mapped pinned: kStagingBuffers head images
    size_t staging_stride = 0;
    volatile int32_t *staging_busy = nullptr;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<int64_t> pending;
    std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;
    int64_t next_ticket = 1;
    int64_t submitted = 0, admitted = 0, completed = 0;
    std::thread loop;
    std::atomic<bool> stopping{false};
    std::atomic<bool> stall_heartbeat{false};
    std::atomic<int32_t> error_word{0};
    std::string launch_error;             // the CUDA error that ended a launch (under mu)
};

namespace {

// Default autotuner sample: n = 32..256 with int32 and int64 force matrices.
void default_sample(std::vector<pimqap_instance> &insts, std::vector<pimqap_params> &ps,
                    std::vector<std::vector<int32_t>> &keep) {
    for (int wide = 0; wide < 2; ++wide)
        for (int n = 32; n <= 256; n += 32) {
            std::vector<int32_t> F((size_t)n * n), D((size_t)n * n);
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j) {
                    const int32_t v = (int32_t)((i * 7 + j * 13) % 100) + (wide ? 30000000 : 0);
                    F[(size_t)i * n + j] = (i == j) ? 0 : v;
                    D[(size_t)i * n + j] = (i == j) ? 0 : (int32_t)((i * 11 + j * 5) % 100);
                }
            keep.push_back(std::move(F));
            keep.push_back(std::move(D));
            pimqap_instance in{n, keep[keep.size() - 2].data(), keep.back().data()};
            insts.push_back(in);
            pimqap_params p;
            pimqap_default_params(&p);
            p.replicas = 32;
            p.groups = 1;
            p.max_megaiters = 500;
            ps.push_back(p);
        }
}

// Slot-sized device and mapped state of one class, and the link of its resident launch.
pimqap_status open_class(Server &S, ServeClass &C) {
    const int m = C.slots;
    C.qcap = 1;
    while (C.qcap < (size_t)m * PIMQAP_MAX_REPLICAS + 1) C.qcap <<= 1;
    C.inbox_cap = 1;
    while (C.inbox_cap < (unsigned)m * 2) C.inbox_cap <<= 1;
    C.done_cap = C.inbox_cap;
    const size_t dbytes = carve_size(sizeof(SolveDev) * m) + 4 * carve_size(8 * (size_t)m) +
                          2 * carve_size(8 * C.qcap) + 8 * carve_size(8);
    PQ_CUDA(cudaMalloc(&C.dbase, dbytes));
    PQ_CUDA(cudaMemset(C.dbase, 0, dbytes));
    char *cur = C.dbase;
    C.d_inst = carve<SolveDev>(cur, m);
    C.d_sym = reinterpret_cast<int32_t *>(carve<int64_t>(cur, m));
    C.d_maxm = carve<int64_t>(cur, m);
    unsigned int *d_finish = reinterpret_cast<unsigned int *>(carve<int64_t>(cur, m));
    carve<int64_t>(cur, m);
    unsigned long long *d_items = carve<unsigned long long>(cur, C.qcap);
    unsigned long long *d_seq = carve<unsigned long long>(cur, C.qcap);
    unsigned long long *d_head = carve<unsigned long long>(cur, 1);
    unsigned long long *d_tail = carve<unsigned long long>(cur, 1);
    int32_t *d_active = reinterpret_cast<int32_t *>(carve<int64_t>(cur, 1));
    int32_t *d_error = reinterpret_cast<int32_t *>(carve<int64_t>(cur, 1));
    unsigned long long *d_start = carve<unsigned long long>(cur, 1);
    unsigned long long *d_inbox_head = carve<unsigned long long>(cur, 1);
    unsigned long long *d_done_tail = carve<unsigned long long>(cur, 1);

    // mapped block: inbox | done | done_seq | flags | descriptors | results | perms | energies
    const size_t ring_words = (size_t)C.inbox_cap + 2 * C.done_cap + 8;
    const size_t ring_bytes = 8 * ring_words + 4 * (size_t)kMaxResidentCtas;
    const size_t desc_off = carve_size(ring_bytes);
    const size_t res_off = desc_off + carve_size(sizeof(ServeDesc) * m);
    const size_t perm_off = res_off + carve_size(sizeof(BatchResultDev) * m);
    const size_t energy_off = perm_off + carve_size(4 * (size_t)m * PIMQAP_MAX_N);
    const size_t hbytes = energy_off + carve_size(8 * (size_t)m * kServeMaxReplicas);
    PQ_CUDA(cudaHostAlloc(&C.hbase, hbytes, cudaHostAllocMapped));
    std::memset(C.hbase, 0, hbytes);
    unsigned long long *h = reinterpret_cast<unsigned long long *>(C.hbase);
    C.h_inbox = h;
    C.h_done = h + C.inbox_cap;
    C.h_done_seq = h + C.inbox_cap + C.done_cap;
    C.h_inbox_tail = h + C.inbox_cap + 2 * C.done_cap;
    C.h_heartbeat = h + C.inbox_cap + 2 * C.done_cap + 1;
    C.h_shutdown = reinterpret_cast<volatile int32_t *>(h + C.inbox_cap + 2 * C.done_cap + 2);
    C.h_error = reinterpret_cast<volatile int32_t *>(h + C.inbox_cap + 2 * C.done_cap + 3);
    C.h_resident = reinterpret_cast<volatile int32_t *>(h + ring_words);
    C.h_desc = reinterpret_cast<volatile ServeDesc *>(C.hbase + desc_off);
    C.h_res = reinterpret_cast<volatile BatchResultDev *>(C.hbase + res_off);
    C.h_perm = reinterpret_cast<volatile int32_t *>(C.hbase + perm_off);
    C.h_energy = reinterpret_cast<volatile long long *>(C.hbase + energy_off);
    void *dev_h = nullptr, *dev_staging = nullptr, *dev_busy = nullptr;
    PQ_CUDA(cudaHostGetDevicePointer(&dev_h, C.hbase, 0));
    PQ_CUDA(cudaHostGetDevicePointer(&dev_staging, S.staging, 0));
    PQ_CUDA(cudaHostGetDevicePointer(&dev_busy, const_cast<int32_t *>(S.staging_busy), 0));
    char *dh = reinterpret_cast<char *>(dev_h);
    unsigned long long *dq = reinterpret_cast<unsigned long long *>(dh);

    C.free_slots.clear();
    for (int k = m - 1; k >= 0; --k) C.free_slots.push_back(k);
    C.slot_ticket.assign(m, 0);

    BatchDev &B = C.B;
    B = BatchDev{};
    B.inst = C.d_inst; B.sym = C.d_sym; B.max_megaiters = C.d_maxm; B.finish_inst = d_finish;
    B.count = m; B.q_items = d_items; B.q_seq = d_seq; B.q_head = d_head; B.q_tail = d_tail;
    B.qmask = (unsigned)C.qcap - 1; B.active = d_active; B.error = d_error; B.start_ns = d_start;
    B.shutdown = reinterpret_cast<volatile int32_t *>(dq + C.inbox_cap + 2 * C.done_cap + 2);
    B.serving = 1;
    ServeLink &L = B.link;
    L.inbox = dq;
    L.inbox_tail = dq + C.inbox_cap + 2 * C.done_cap;
    L.inbox_head = d_inbox_head;
    L.inbox_mask = C.inbox_cap - 1;
    L.desc = reinterpret_cast<const volatile ServeDesc *>(dh + desc_off);
    L.staging = reinterpret_cast<const unsigned char *>(dev_staging);
    L.staging_stride = S.staging_stride;
    L.staging_busy = reinterpret_cast<volatile int32_t *>(dev_busy);
    L.results = reinterpret_cast<volatile BatchResultDev *>(dh + res_off);
    L.result_perm = reinterpret_cast<volatile int32_t *>(dh + perm_off);
    L.result_energy = reinterpret_cast<volatile long long *>(dh + energy_off);
    L.energy_stride = kServeMaxReplicas;
    L.done = dq + C.inbox_cap;
    L.done_seq = dq + C.inbox_cap + C.done_cap;
    L.done_tail = d_done_tail;
    L.done_mask = C.done_cap - 1;
    L.heartbeat = dq + C.inbox_cap + 2 * C.done_cap + 1;
    L.heartbeat_limit_ns =
        (unsigned long long)((S.cfg.heartbeat_timeout_s > 0 ? S.cfg.heartbeat_timeout_s : 10.0) * 1e9);
    L.error_host = reinterpret_cast<volatile int32_t *>(dq + C.inbox_cap + 2 * C.done_cap + 3);
    L.resident = reinterpret_cast<volatile int32_t *>(dq + ring_words);
    L.inst_rw = C.d_inst;
    L.sym_rw = C.d_sym;
    L.maxm_rw = C.d_maxm;
    B.worker_threads = C.shape.worker_threads;
    B.workers = C.shape.workers;
    B.slice_bytes = (unsigned)C.shape.slice;
    PQ_CUDA(cudaStreamCreateWithFlags(&C.stream, cudaStreamNonBlocking));
    return PIMQAP_OK;
}

// The class that runs a request most cheaply: exact force width first, then the smallest
// cluster and slice that fit.  The request is re-planned for that class's width and cluster.
// Whether an instance needing `bits`-wide forces can run in a launch of shape sh (and its
// plan there, in *out).
bool class_fits(const BatchClass &sh, const pimqap_instance &inst, const pimqap_params &params,
                const InstanceInfo &info, int bits, int maxsm, Plan *out = nullptr) {
    if (sh.bits < bits) return false;
    pimqap_params p = params;
    p.force_bits = sh.bits;
    Plan P;
    if (plan_instance(&inst, &p, (size_t)maxsm, sh.cl, &P, &info) != PIMQAP_OK) return false;
    const size_t need = sh.cl == 1 ? pimqap::batch_slice_bytes(P.n, sh.bits)
                                    : 16 + std::max(P.smem, pimqap::exchange_scratch_bytes());
    if (need > sh.slice) return false;
    if ((P.n + sh.worker_threads - 1) / sh.worker_threads > 4) return false;   // candidates per lane
    if (out) *out = P;
    return true;
}

// Replica workers of a launch: replicas it runs at once.
size_t class_workers(const BatchClass &sh) {
    return sh.cl == 1 ? (size_t)sh.grid * sh.workers : (size_t)(sh.grid / sh.cl);
}

// The class a request joins: among the launches it fits, the one expected to finish it first:
// the work already routed there spread over its workers, plus the request's own work spread
// over the workers it can use (one per replica).  The request's cost is added to that class's
// load (under S.mu) until it completes.
int route(Server &S, Request &R) {
    std::vector<std::pair<int, double>> fits;
    for (int c = 0; c < (int)S.classes.size(); ++c) {
        Plan P;
        if (!class_fits(S.classes[c].shape, R.inst, R.params, R.info, R.plan.bits, S.maxsm, &P)) continue;
        fits.push_back({c, instance_work(P, std::min<int64_t>(R.params.max_megaiters, 1000000))});
    }
    const double reps = (double)R.plan.T * R.plan.R;
    std::lock_guard<std::mutex> lk(S.mu);
    int best = -1;
    double best_cost = 1e300;
    for (const auto &f : fits) {
        const ServeClass &C = S.classes[f.first];
        const double W = (double)std::max<size_t>(1, class_workers(C.shape));
        const double cost = C.load / W + f.second / std::min(reps, W);
        if (cost < best_cost) {
            best_cost = cost;
            best = f.first;
        }
    }
    if (best >= 0) {
        for (const auto &f : fits)
            if (f.first == best) R.work = f.second;
        S.classes[best].load += R.work;
    }
    return best;
}

// The finished request's result from its class's mapped result slot.
void read_result(Server &S, Request &R) {
    ServeClass &C = S.classes[R.cls];
    const Plan &P = R.plan;
    const size_t reps = (size_t)P.T * P.R;
    volatile BatchResultDev &o = C.h_res[R.slot];
    pimqap_result &res = R.result;
    std::memset(&res, 0, sizeof(res));
    R.perm.resize(P.n);
    for (int q = 0; q < P.n; ++q) R.perm[q] = C.h_perm[(size_t)R.slot * PIMQAP_MAX_N + q];
    R.energies.resize(reps);
    for (size_t r = 0; r < reps; ++r) R.energies[r] = C.h_energy[(size_t)R.slot * kServeMaxReplicas + r];
    res.best_energy = std::min<int64_t>(o.best, o.single_best);
    res.target_megaiter = (o.target_epoch == std::numeric_limits<long long>::max()) ? -1 : o.target_epoch;
    res.megaiters_done = o.epoch;
    res.updates = (int64_t)o.epoch * P.spe * P.n * (int64_t)reps;
    res.sweeps = res.updates / P.n;
    res.proposals = res.sweeps * ((int64_t)P.n * (P.n - 1) / 2);
    res.accepts = (int64_t)o.accepts;
    res.force_bits = P.bits;
    res.cluster_size = P.cl;
    res.stopped_by = (o.stop_epoch != pimqap::kNoStop) ? 1 : 0;
    res.h2d_bytes = (int64_t)P.head;
    res.d2h_bytes = (int64_t)(sizeof(BatchResultDev) + 4 * (size_t)P.n + 8 * reps);
    res.beta_max_used = R.params.beta_internal ? R.params.beta_max : R.params.beta_max * 1.44269504089;
    res.beta_ratio_used = R.params.beta_ratio;
    R.status = o.error ? PIMQAP_ERR_DEVICE : PIMQAP_OK;
}

void release(Server &S, Request &R) {
    ServeClass &C = S.classes[R.cls];
    S.arena.release(R.off, R.plan.total);
    C.free_slots.push_back(R.slot);
    C.slot_ticket[R.slot] = 0;
    C.replicas_in_flight -= (size_t)R.plan.T * R.plan.R;
    C.load = std::max(0.0, C.load - R.work);
}

// One pass of admissions in arrival order: every pending request whose class has a free slot
// and queue room, for which the arena has memory and a staging buffer is free.
bool admit_some(Server &S) {
    bool any = false;
    std::lock_guard<std::mutex> lk(S.mu);
    for (auto it = S.pending.begin(); it != S.pending.end();) {
        Request &R = *S.reqs[*it];
        ServeClass &C = S.classes[R.cls];
        const size_t reps = (size_t)R.plan.T * R.plan.R;
        int stg = -1;
        for (int b = 0; b < kStagingBuffers; ++b)
            if (S.staging_busy[b] == 0) {
                stg = b;
                break;
            }
        if (stg < 0) break;
        size_t off = 0;
        // About two rounds of the launch's workers in flight at most: the queue serves the
        // admitted instances' epochs in turn, so admitting more only spreads the workers over
        // more requests and delays them all (the rest wait here, in arrival order).
        const bool crowded = C.replicas_in_flight >= 2 * class_workers(C.shape);
        if (C.free_slots.empty() || crowded || C.replicas_in_flight + reps > C.qcap - 1 ||
            !S.arena.alloc(R.plan.total, &off)) {
            ++it;
            continue;
        }
        R.off = off;
        R.slot = C.free_slots.back();
        C.free_slots.pop_back();
        C.slot_ticket[R.slot] = R.ticket;
        C.replicas_in_flight += reps;
        const Plan &P = R.plan;
        char *base = S.arena_base + R.off;
        carve_instance(P, base, base + P.head, &R.dev);
        R.dev.goal = R.params.goal;
        R.dev.seed = R.params.seed;
        fill_head(&R.inst, &R.params, P, S.staging + (size_t)stg * S.staging_stride);
        volatile ServeDesc &d = C.h_desc[R.slot];
        ServeDesc tmp{};
        tmp.dev = R.dev;
        tmp.max_megaiters = R.params.max_megaiters;
        tmp.head_bytes = P.head;
        tmp.tail_bytes = P.tail;
        tmp.sym = P.sym ? 1 : 0;
        tmp.bits = P.bits;
        std::memcpy(const_cast<ServeDesc *>(&d), &tmp, sizeof(tmp));
        S.staging_busy[stg] = 1;
        std::atomic_thread_fence(std::memory_order_seq_cst);
        C.h_inbox[C.inbox_tail & (C.inbox_cap - 1)] = ((unsigned long long)R.slot << 32) | (unsigned)stg;
        std::atomic_thread_fence(std::memory_order_seq_cst);
        *C.h_inbox_tail = ++C.inbox_tail;
        std::atomic_thread_fence(std::memory_order_seq_cst);
        R.state = Request::kRunning;
        R.t_admit = Clock::now();
        ++S.admitted;
        it = S.pending.erase(it);
        any = true;
    }
    return any;
}

bool complete_some(Server &S) {
    bool any = false;
    for (auto &C : S.classes) {
        for (;;) {
            const unsigned long long h = C.done_head;
            if (C.h_done_seq[h & (C.done_cap - 1)] != h + 1) break;
            std::atomic_thread_fence(std::memory_order_seq_cst);
            const int slot = (int)C.h_done[h & (C.done_cap - 1)];
            C.done_head = h + 1;
            std::lock_guard<std::mutex> lk(S.mu);
            Request &R = *S.reqs[C.slot_ticket[slot]];
            read_result(S, R);
            release(S, R);
            R.t_done = Clock::now();
            R.state = R.status == PIMQAP_OK ? Request::kDone : Request::kFailed;
            ++S.completed;
            S.cv.notify_all();
            any = true;
        }
    }
    return any;
}

// The server thread: no work is enqueued while the resident launches run (the only CUDA
// call is a periodic stream query, which enqueues nothing): a launch that ended while serving
// (a device fault ends them all) sets kErrLaunchEnded, so waiters fail instead of waiting.
void serve_loop(Server *S) {
    unsigned long long beat = 1;
    auto last_query = Clock::now();
    for (;;) {
        if (!S->stall_heartbeat.load())
            for (auto &C : S->classes) *C.h_heartbeat = ++beat;
        int32_t err = 0;
        for (auto &C : S->classes) err |= *C.h_error;
        if (std::chrono::duration<double>(Clock::now() - last_query).count() > 0.05) {
            last_query = Clock::now();
            for (size_t k = 0; k < S->classes.size(); ++k) {
                const cudaError_t q = cudaStreamQuery(S->classes[k].stream);
                if (q == cudaErrorNotReady) continue;
                err |= pimqap::kErrLaunchEnded;
                std::lock_guard<std::mutex> lk(S->mu);
                if (S->launch_error.empty())
                    S->launch_error = "serving launch " + std::to_string(k) + " ended: " + cudaGetErrorString(q);
            }
        }
        if (err && (S->error_word.load() | err) != S->error_word.load()) {
            S->error_word.fetch_or(err);
            std::lock_guard<std::mutex> lk(S->mu);
            S->cv.notify_all();
        }
        bool busy = complete_some(*S);
        busy |= admit_some(*S);
        if (S->stopping.load()) break;   // destroy: running requests are abandoned
        if (!busy) std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
}

void fill_out(const Request &R, pimqap_result *out) {
    int32_t *perm_dst = out->best_perm;
    int64_t *energy_dst = out->final_energies;
    *out = R.result;
    out->best_perm = perm_dst;
    out->final_energies = energy_dst;
    if (perm_dst && !R.perm.empty()) std::memcpy(perm_dst, R.perm.data(), 4 * R.perm.size());
    if (energy_dst && !R.energies.empty()) std::memcpy(energy_dst, R.energies.data(), 8 * R.energies.size());
    out->admit_ms = std::chrono::duration<double, std::milli>(R.t_admit - R.t_submit).count();
    out->latency_ms = std::chrono::duration<double, std::milli>(R.t_done - R.t_submit).count();
    out->wall_ms = out->latency_ms;
}

}  // namespace
}  // namespace detail
}  // namespace pimqap

using namespace pimqap::detail;

struct pimqap_server {
    Server s;
};

extern "C" {

pimqap_status pimqap_server_create(const pimqap_server_config *config, pimqap_server **out) {
    if (!config || !out) return fail(PIMQAP_ERR_ARG, "null config or handle");
    *out = nullptr;
    auto h = std::unique_ptr<pimqap_server>(new pimqap_server());
    Server &S = h->s;
    S.cfg = *config;
    S.device = config->device;
    pimqap_status st = open_device(S.device, &S.maxsm);
    if (st != PIMQAP_OK) return st;
    PQ_CUDA(cudaDeviceGetAttribute(&S.sms, cudaDevAttrMultiProcessorCount, S.device));
    // autotuner: classes and SM shares from the sample
    std::vector<pimqap_instance> sample;
    std::vector<pimqap_params> sparams;
    std::vector<std::vector<int32_t>> keep;
    if (config->sample && config->sample_params && config->sample_count > 0) {
        sample.assign(config->sample, config->sample + config->sample_count);
        sparams.assign(config->sample_params, config->sample_params + config->sample_count);
    } else {
        default_sample(sample, sparams, keep);
    }
    std::vector<Plan> plans(sample.size());
    std::vector<int64_t> megaiters(sample.size());
    for (size_t k = 0; k < sample.size(); ++k) {
        st = check_params(&sample[k], &sparams[k]);
        if (st != PIMQAP_OK) return st;
        st = plan_instance(&sample[k], &sparams[k], (size_t)S.maxsm, sparams[k].cluster_size, &plans[k]);
        if (st != PIMQAP_OK) return st;
        megaiters[k] = sparams[k].max_megaiters;
    }
    std::vector<BatchClass> shapes = plan_classes(plans, megaiters, S.sms, S.maxsm, 0);
    if (autotune_enabled()) {   // worker shapes measured on the sample (one mega-iteration each)
        st = tune_classes(sample.data(), sparams.data(), (int32_t)sample.size(), plans, shapes, S.sms,
                          S.maxsm, nullptr, true);
        if (st != PIMQAP_OK) return st;
    }
    if (config->sample && config->sample_count > 0) {
        // Every shape a request can have (n <= PIMQAP_MAX_N, int32 or int64 forces) must find a
        // resident launch: shapes of the built-in sample that no class from the caller's sample
        // fits get a class of their own, with the smallest SM share.
        std::vector<pimqap_instance> dsample;
        std::vector<pimqap_params> dparams;
        std::vector<std::vector<int32_t>> dkeep;
        default_sample(dsample, dparams, dkeep);
        std::vector<Plan> missing;
        std::vector<int64_t> mmega;
        for (size_t k = 0; k < dsample.size(); ++k) {
            const InstanceInfo info = analyse(dsample[k].n, dsample[k].flow, dsample[k].dist);
            Plan P;
            st = plan_instance(&dsample[k], &dparams[k], (size_t)S.maxsm, 0, &P, &info);
            if (st != PIMQAP_OK) return st;
            bool fits = false;
            for (const auto &c : shapes) fits = fits || class_fits(c, dsample[k], dparams[k], info, P.bits, S.maxsm);
            if (!fits) {
                missing.push_back(P);
                mmega.push_back(1);
            }
        }
        if (!missing.empty()) {
            std::vector<BatchClass> extra = plan_classes(missing, mmega, S.sms, S.maxsm, 0);
            for (auto &c : extra) {
                c.work = 0;
                c.members.clear();
                shapes.push_back(c);
            }
        }
    }
    // Resident side by side: each class gets a share of the SMs by work and one CTA per SM of
    // its share.  With no more CTAs than SMs in total, every CTA finds an SM it fits alone,
    // so no class is left without resident workers.  Cluster classes launch first.
    std::stable_sort(shapes.begin(), shapes.end(),
                     [](const BatchClass &a, const BatchClass &b) { return a.cl > b.cl; });
    double total = 0;
    for (auto &c : shapes) total += c.work;
    // SMs left to the server's own short kernels (set-up of admitted requests, result gather):
    // the resident launches never release theirs.
    constexpr int kReservedSms = 4;
    const int sms_for_classes = S.sms - kReservedSms;
    int sm_left = sms_for_classes;
    int min_need = 0;
    for (auto &c : shapes) min_need += c.cl;
    if (min_need > sms_for_classes) return fail(PIMQAP_ERR_ARG, "too many serving classes for this GPU");
    for (size_t k = 0; k < shapes.size(); ++k) {
        BatchClass &c = shapes[k];
        int rest = 0;
        for (size_t q = k + 1; q < shapes.size(); ++q) rest += shapes[q].cl;
        int share = (int)std::lround(total > 0 ? c.work / total * sms_for_classes
                                               : (double)sms_for_classes / shapes.size());
        share = std::max(c.cl, std::min(share, sm_left - rest));
        share -= share % c.cl;
        sm_left -= share;
        c.grid = share;
    }
    S.classes.resize(shapes.size());
    const int slots = config->slots_per_class > 0 ? config->slots_per_class : 128;
    // arena inside the memory budget
    size_t free_b = 0, total_b = 0;
    PQ_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t budget = config->memory_budget_bytes > 0 ? (size_t)config->memory_budget_bytes : free_b / 2;
    PQ_CUDA(cudaMalloc(&S.arena_base, budget));
    S.arena.reset(budget);
    // staging pool (mapped): head images of requests being admitted
    S.staging_stride = carve_size(4 * carve_size((size_t)PIMQAP_MAX_N * PIMQAP_MAX_N * 4) +
                                  2 * carve_size(4 * PIMQAP_MAX_N) +
                                  carve_size((size_t)kServeMaxReplicas * PIMQAP_MAX_N * 4) +
                                  carve_size((size_t)kServeMaxReplicas * 8) + carve_size((size_t)kServeMaxRankSlots * 4) +
                                  carve_size(kServeMaxReplicas * 8) + 4 * carve_size(8));
    PQ_CUDA(cudaHostAlloc(&S.staging, S.staging_stride * kStagingBuffers + 256, cudaHostAllocMapped));
    int32_t *busy = nullptr;
    PQ_CUDA(cudaHostAlloc(&busy, 4 * kStagingBuffers, cudaHostAllocMapped));
    std::memset(busy, 0, 4 * kStagingBuffers);
    S.staging_busy = busy;
    for (size_t k = 0; k < shapes.size(); ++k) {
        S.classes[k].shape = shapes[k];
        S.classes[k].slots = slots;
        st = open_class(S, S.classes[k]);
        if (st != PIMQAP_OK) return st;
    }
    PQ_CUDA(cudaDeviceSynchronize());
    // every buffer exists: now the resident launches, cluster classes first, each one only
    // after every CTA of the previous one has started (launches on different streams may be
    // placed in any order, and CTAs of a later launch could take the SMs a cluster needs)
    unsigned long long beat = 1;
    for (size_t k = 0; k < S.classes.size(); ++k) {
        ServeClass &C = S.classes[k];
        PQ_CUDA(pimqap::launch_batch(C.B, C.shape.bits, C.shape.cl, C.shape.grid, C.stream));
        const auto t0 = Clock::now();
        for (;;) {
            int up = 0;
            for (int b = 0; b < C.shape.grid; ++b) up += C.h_resident[b] ? 1 : 0;
            if (up == C.shape.grid) break;
            for (size_t q = 0; q <= k; ++q) *S.classes[q].h_heartbeat = ++beat;
            if (std::chrono::duration<double>(Clock::now() - t0).count() > 10.0) {
                const std::string why = "serving launch " + std::to_string(k) + " (" +
                                        std::to_string(C.shape.grid) + " CTAs, cluster " +
                                        std::to_string(C.shape.cl) + ") did not become resident";
                pimqap_server_destroy(h.release());
                return fail(PIMQAP_ERR_CUDA, why);
            }
            std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
    }
    S.loop = std::thread(serve_loop, &S);
    *out = h.release();
    return PIMQAP_OK;
}

pimqap_status pimqap_server_submit(pimqap_server *h, const pimqap_instance *inst,
                                   const pimqap_params *params, int64_t *ticket) {
    if (!h || !ticket) return fail(PIMQAP_ERR_ARG, "null server or ticket");
    Server &S = h->s;
    pimqap_status st = check_params(inst, params);
    if (st != PIMQAP_OK) return st;
    if (params->active_facilities > 0)
        return fail(PIMQAP_ERR_ARG, "active_facilities is supported by pimqap_solve and solver handles only");
    if (params->update_rule != PIMQAP_RULE_SEQUENTIAL)
        return fail(PIMQAP_ERR_ARG, "the one-shot rule is supported by pimqap_solve and solver handles only");
    if (params->auto_beta) return fail(PIMQAP_ERR_ARG, "automatic beta selection needs pimqap_solve");
    if ((int64_t)params->groups * params->replicas > kServeMaxReplicas)
        return fail(PIMQAP_ERR_ARG, "a served request holds at most 1024 replicas (groups x replicas)");
    {
        const int64_t cap = params->rank_slots ? params->rank_slots : std::max(params->replicas, 10);
        if ((int64_t)params->groups * cap > kServeMaxRankSlots)
            return fail(PIMQAP_ERR_ARG, "groups x rank slots too large for serving");
    }
    if (S.error_word.load()) {
        std::lock_guard<std::mutex> lk(S.mu);
        return fail(PIMQAP_ERR_DEVICE, "the server's device launches stopped (error word " +
                                           std::to_string(S.error_word.load()) + ") " + S.launch_error);
    }
    auto R = std::unique_ptr<Request>(new Request());
    const int n = inst->n;
    R->F.assign(inst->flow, inst->flow + (size_t)n * n);
    R->D.assign(inst->dist, inst->dist + (size_t)n * n);
    R->inst = pimqap_instance{n, R->F.data(), R->D.data()};
    R->params = *params;
    R->params.device = S.device;
    R->info = analyse(n, R->inst.flow, R->inst.dist);
    st = plan_instance(&R->inst, &R->params, (size_t)S.maxsm, 0, &R->plan, &R->info);
    if (st != PIMQAP_OK) return st;
    R->cls = route(S, *R);
    if (R->cls < 0) return fail(PIMQAP_ERR_BUSY, "no resident launch fits this request's shape");
    pimqap_params p = R->params;
    p.force_bits = S.classes[R->cls].shape.bits;
    st = plan_instance(&R->inst, &p, (size_t)S.maxsm, S.classes[R->cls].shape.cl, &R->plan, &R->info);
    if (st != PIMQAP_OK) return st;
    R->params.force_bits = p.force_bits;
    if (carve_size(R->plan.total) > S.arena.size()) {
        {
            std::lock_guard<std::mutex> lk(S.mu);
            S.classes[R->cls].load = std::max(0.0, S.classes[R->cls].load - R->work);
        }
        return fail(PIMQAP_ERR_BUSY, "request needs " + std::to_string(R->plan.total) +
                                         " bytes of device memory; the budget is " +
                                         std::to_string(S.arena.size()));
    }
    R->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(S.mu);
    R->ticket = S.next_ticket++;
    *ticket = R->ticket;
    S.pending.push_back(R->ticket);
    S.reqs[R->ticket] = std::move(R);
    ++S.submitted;
    return PIMQAP_OK;
}

pimqap_status pimqap_server_poll(pimqap_server *h, int64_t ticket, pimqap_result *result) {
    return pimqap_server_wait(h, ticket, 0.0, result);
}

pimqap_status pimqap_server_wait(pimqap_server *h, int64_t ticket, double timeout_s,
                                 pimqap_result *result) {
    if (!h || !result) return fail(PIMQAP_ERR_ARG, "null server or result");
    Server &S = h->s;
    std::unique_lock<std::mutex> lk(S.mu);
    auto it = S.reqs.find(ticket);
    if (it == S.reqs.end()) return fail(PIMQAP_ERR_ARG, "unknown ticket");
    auto ready = [&] {
        const Request &R = *S.reqs[ticket];
        return R.state == Request::kDone || R.state == Request::kFailed || S.error_word.load() != 0;
    };
    if (timeout_s < 0) S.cv.wait(lk, ready);
    else if (timeout_s > 0) S.cv.wait_for(lk, std::chrono::duration<double>(timeout_s), ready);
    Request &R = *S.reqs[ticket];
    if (R.state == Request::kFailed) {
        const pimqap_status st = R.status;
        S.reqs.erase(ticket);
        return fail(st, "served request failed");
    }
    if (R.state != Request::kDone) {
        if (S.error_word.load())
            return fail(PIMQAP_ERR_DEVICE, "the server's device launches stopped (error word " +
                                               std::to_string(S.error_word.load()) + ") " + S.launch_error);
        return fail(PIMQAP_ERR_NOT_READY, "request not finished");
    }
    fill_out(R, result);
    S.reqs.erase(ticket);
    return PIMQAP_OK;
}

pimqap_status pimqap_server_stats_get(pimqap_server *h, pimqap_server_stats *stats) {
    if (!h || !stats) return fail(PIMQAP_ERR_ARG, "null server or stats");
    Server &S = h->s;
    std::lock_guard<std::mutex> lk(S.mu);
    stats->submitted = S.submitted;
    stats->admitted = S.admitted;
    stats->completed = S.completed;
    stats->pending = (int64_t)S.pending.size();
    stats->memory_in_use = (int64_t)S.arena.used();
    stats->memory_budget = (int64_t)S.arena.size();
    stats->classes = (int32_t)S.classes.size();
    stats->error_word = S.error_word.load();
    return PIMQAP_OK;
}

void pimqap_server_destroy(pimqap_server *h) {
    if (!h) return;
    Server &S = h->s;
    {
        std::lock_guard<std::mutex> lk(S.mu);
        if (std::getenv("PIMQAP_TRACE")) {   // state of every class at shutdown
            std::vector<int> pend(S.classes.size(), 0);
            for (int64_t t : S.pending) ++pend[S.reqs[t]->cls];
            int busy = 0;
            for (int b = 0; b < kStagingBuffers; ++b) busy += S.staging_busy[b] ? 1 : 0;
            std::fprintf(stderr, "[pimqap] server: %zu pending, %d staging buffers busy, error word %d %s\n",
                         S.pending.size(), busy, S.error_word.load(), S.launch_error.c_str());
            for (size_t k = 0; k < S.classes.size(); ++k) {
                const ServeClass &C = S.classes[k];
                std::fprintf(stderr, "[pimqap] class %zu bits=%d cl=%d band=%d grid=%d workers=%d: load %.3g, "
                                     "replicas in flight %zu, free slots %zu/%d, pending %d, inbox %llu\n",
                             k, C.shape.bits, C.shape.cl, C.shape.band, C.shape.grid, C.shape.workers, C.load,
                             C.replicas_in_flight, C.free_slots.size(), C.slots, pend[k], C.inbox_tail);
            }
        }
        S.pending.clear();
    }
    S.stopping.store(true);
    if (S.loop.joinable()) S.loop.join();
    unsigned long long beat = 1ull << 62;
    bool inflight = false;
    for (auto &C : S.classes)
        if (C.replicas_in_flight) inflight = true;
    for (auto &C : S.classes) {
        // drain when nothing is in flight; leave at once (abandoning running requests) when
        // something is, or after a device error
        if (C.h_shutdown) *C.h_shutdown = (inflight || S.error_word.load()) ? 2 : 1;
        std::atomic_thread_fence(std::memory_order_seq_cst);
    }
    // keep beating until every class's workers have seen the shutdown and left; only then
    // free anything (freeing can synchronise the device)
    for (;;) {
        bool running = false;
        for (auto &C : S.classes)
            if (C.stream && cudaStreamQuery(C.stream) == cudaErrorNotReady) running = true;
        if (!running) break;
        for (auto &D : S.classes) *D.h_heartbeat = ++beat;
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
    if (std::getenv("PIMQAP_TRACE")) {   // where every abandoned request had got to
        for (auto &kv : S.reqs) {
            const Request &R = *kv.second;
            if (R.state != Request::kRunning) continue;
            int32_t e = -1, err = 0;
            const cudaError_t c1 = cudaMemcpy(&e, R.dev.epoch, 4, cudaMemcpyDeviceToHost);
            cudaMemcpy(&err, R.dev.error, 4, cudaMemcpyDeviceToHost);
            if (c1 != cudaSuccess) std::fprintf(stderr, "[pimqap] read-back: %s\n", cudaGetErrorString(c1));
            const double age = std::chrono::duration<double>(Clock::now() - R.t_admit).count();
            std::fprintf(stderr, "[pimqap] running ticket %lld class %d slot %d n=%d reps=%d: epoch %d of %lld, "
                                 "error %d, admitted %.1f s ago\n",
                         (long long)R.ticket, R.cls, R.slot, R.plan.n, R.plan.T * R.plan.R, e,
                         (long long)R.params.max_megaiters, err, age);
        }
    }
    for (auto &C : S.classes) {
        if (C.stream) cudaStreamDestroy(C.stream);
        if (C.dbase) cudaFree(C.dbase);
        if (C.hbase) cudaFreeHost(C.hbase);
    }
    if (S.arena_base) cudaFree(S.arena_base);
    if (S.staging) cudaFreeHost(S.staging);
    if (S.staging_busy) cudaFreeHost(const_cast<int32_t *>(S.staging_busy));
    delete h;
}

// Host-side fault injection for tests: stall (1) or resume (0) the server thread's heartbeat.
void pimqap_server_debug_stall_heartbeat(pimqap_server *h, int32_t stall) {
    if (h) h->s.stall_heartbeat.store(stall != 0);
}

}  // extern "C"
