// pimqap_batch.cpp - batched solve: many independent instances of uneven n in persistent
// launches (no reference counterpart: the reference solves one instance per process).
//
// A batch is partitioned into classes: force-matrix width x CTAs per replica (1, 2 or 4) x,
// for single-CTA replicas, a band of n.  Each class is one persistent launch whose workers (a
// group of warps with its own named barrier and shared-memory slice, or a whole cluster) pop
// replica-epochs from a device queue.  The classes run concurrently on separate streams, each
// with a grid that fills the GPU, largest class first.  The autotuner (tune_classes) times one
// mega-iteration of a class's instances under each candidate worker shape - threads per
// replica and replicas (workers) per CTA - and keeps the fastest; the choice is cached per
// class shape for the rest of the process.  Results are gathered on the device and read back
// in one copy per class.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <string>
#include <thread>
#include <vector>

#include "pimqap.h"
#include "pimqap_batch.h"
#include "pimqap_internal.h"
#include "pimqap_plan.h"

namespace pimqap {
namespace detail {

namespace {

// n bands of single-CTA classes: small n packs more workers into a CTA.
constexpr int kBandEdges[] = {48, 96, 160, 256};

int band_of(int n) {
    int b = 0;
    while (n > kBandEdges[b]) ++b;
    return b;
}

}  // namespace

double instance_work(const Plan &P, int64_t megaiters) {
    // updates x (candidate deltas + an expected share of the n^2 force update)
    const double upd = (double)P.T * P.R * (double)megaiters * P.spe * P.n;
    return upd * ((double)P.n + 0.25 * (double)P.n * P.n / 8.0);
}

std::vector<BatchClass> plan_classes(const std::vector<Plan> &plans, const std::vector<int64_t> &megaiters,
                                     int sms, int maxsm, int force_cluster) {
    std::vector<BatchClass> classes;
    auto find = [&](int bits, int cl, int band) -> BatchClass & {
        for (auto &c : classes)
            if (c.bits == bits && c.cl == cl && c.band == band) return c;
        classes.push_back(BatchClass{});
        BatchClass &c = classes.back();
        c.bits = bits;
        c.cl = cl;
        c.band = band;
        return c;
    };
    for (int k = 0; k < (int)plans.size(); ++k) {
        const Plan &P = plans[k];
        const bool single = P.cl == 1 && pimqap::batch_slice_bytes(P.n, P.bits) <= (size_t)maxsm && !force_cluster;
        BatchClass &c = find(P.bits, single ? 1 : P.cl, single ? band_of(P.n) : 0);
        c.members.push_back(k);
        c.work += instance_work(P, megaiters[k]);
    }
    for (auto &c : classes) {
        c.nmax = 0;
        for (int k : c.members) c.nmax = std::max(c.nmax, plans[k].n);
        int nmax = 0;
        size_t slice = 0;
        for (int k : c.members) {
            const Plan &P = plans[k];
            nmax = std::max(nmax, P.n);
            slice = std::max(slice, c.cl == 1 ? pimqap::batch_slice_bytes(P.n, c.bits)
                                               : 16 + std::max(P.smem, pimqap::exchange_scratch_bytes()));
        }
        c.slice = (slice + 15) & ~size_t(15);
        if (c.cl == 1) {
            c.worker_threads = nmax <= 32 ? 32 : (nmax <= 64 ? 64 : 128);
            c.workers = std::max(1, std::min(256 / c.worker_threads, (int)((size_t)maxsm / c.slice)));
        } else {
            c.worker_threads = nmax <= 128 * c.cl ? 128 : 256;
            c.workers = 1;
        }
        int occ = 0;
        if (pimqap::batch_occupancy(c.bits, c.cl, c.workers * c.worker_threads, c.workers * c.slice, &occ) !=
                cudaSuccess || occ < 1)
            occ = 1;
        // Every class gets a grid that fills the GPU: classes are launched largest first on
        // their own streams, and a class's CTAs start on the SMs the previous classes' workers
        // release when their work runs out.
        c.grid = (c.cl == 1) ? sms * occ : occ * c.cl;   // occ: resident clusters for cl > 1
    }
    std::stable_sort(classes.begin(), classes.end(),
                     [](const BatchClass &a, const BatchClass &b) { return a.work > b.work; });
    return classes;
}

// ------------------------------------------------------------------ the autotuner

namespace {

struct TuneKey {
    int bits, cl, band, nmax16, spe, one_per_sm;
    bool operator<(const TuneKey &o) const {
        return std::tie(bits, cl, band, nmax16, spe, one_per_sm) <
               std::tie(o.bits, o.cl, o.band, o.nmax16, o.spe, o.one_per_sm);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, ClassTuning> g_tune;

TuneKey key_of(const BatchClass &c, const std::vector<Plan> &plans, bool one_per_sm) {
    int spe = 0;
    for (int k : c.members) spe = std::max(spe, plans[k].spe);
    return TuneKey{c.bits, c.cl, c.band, (c.nmax + 15) / 16, spe, one_per_sm ? 1 : 0};
}

// Worker shapes a class can run: threads per replica from 32 to 256 (every lane holds at most
// four candidates, the launch at most 256 threads), as many workers per CTA as shared memory
// and the launch allow.  Cluster classes run one worker per CTA of 128 or 256 threads.
std::vector<std::pair<int, int>> tune_candidates(const BatchClass &c, int maxsm) {
    std::vector<std::pair<int, int>> out;
    for (int wt : {32, 64, 128, 256}) {
        if (c.cl > 1 && wt < 128) continue;
        if ((c.nmax + wt - 1) / wt > 4) continue;
        if (c.cl > 1) {
            out.emplace_back(wt, 1);
            continue;
        }
        for (int w = 1; w * wt <= 256 && (size_t)w * c.slice <= (size_t)maxsm; ++w) out.emplace_back(wt, w);
    }
    return out;
}

// The grid of a shape: every SM filled with as many CTAs (clusters) as fit, or with one CTA
// (cluster) per SM.
int shape_grid(const BatchClass &c, int sms, bool one_per_sm) {
    if (one_per_sm) return (c.cl == 1) ? sms : (sms / c.cl) * c.cl;
    int occ = 0;
    if (pimqap::batch_occupancy(c.bits, c.cl, c.workers * c.worker_threads, c.workers * c.slice, &occ) !=
            cudaSuccess || occ < 1) {
        cudaGetLastError();
        occ = 1;
    }
    return (c.cl == 1) ? sms * occ : occ * c.cl;
}

}  // namespace

bool autotune_enabled() {
    const char *v = std::getenv("PIMQAP_AUTOTUNE");
    return !(v && v[0] == '0');
}

pimqap_status tune_classes(const pimqap_instance *insts, const pimqap_params *params, int32_t count,
                           const std::vector<Plan> &plans, std::vector<BatchClass> &classes, int sms,
                           int maxsm, std::vector<ClassTuning> *report, bool one_per_sm) {
    for (auto &c : classes) {
        const TuneKey key = key_of(c, plans, one_per_sm);
        ClassTuning t{};
        bool cached = false;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto it = g_tune.find(key);
            if (it != g_tune.end()) {
                t = it->second;
                cached = true;
            }
        }
        const auto cands = tune_candidates(c, maxsm);
        int64_t reps = 0;
        for (int k : c.members) reps += (int64_t)plans[k].T * plans[k].R;
        if (!cached && cands.size() > 1 && reps > 0) {
            // one mega-iteration of every member, no goal: the same work under every shape
            std::vector<pimqap_params> tp(params, params + count);
            for (int k : c.members) {
                tp[k].max_megaiters = 1;
                tp[k].goal = std::numeric_limits<int64_t>::min();
                tp[k].timeout_s = 0;
            }
            std::vector<pimqap_result> scratch(count);
            for (auto &r : scratch) std::memset(&r, 0, sizeof(r));
            double work = 0;
            for (int k : c.members) work += instance_work(plans[k], 1);
            t.fixed_threads = c.worker_threads;
            t.fixed_workers = c.workers;
            double best_ms = 0;
            for (const auto &cand : cands) {
                BatchClass cc = c;
                cc.worker_threads = cand.first;
                cc.workers = cand.second;
                cc.grid = shape_grid(cc, sms, one_per_sm);
                ClassRun run;
                pimqap_status st = run.prepare(insts, tp.data(), plans, cc);
                if (st == PIMQAP_OK) st = run.launch();
                if (st == PIMQAP_OK) st = run.finish(plans, scratch.data());
                if (st != PIMQAP_OK) return st;
                const double ms = run.device_ms;
                ++t.tried;
                if (cand.first == c.worker_threads && cand.second == c.workers) t.fixed_ms = ms;
                if (best_ms == 0 || ms < best_ms) {
                    best_ms = ms;
                    t.threads = cand.first;
                    t.workers = cand.second;
                }
            }
            t.tuned_ms = best_ms;
            t.work = work;
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tune[key] = t;
            cached = true;
        }
        // a shape cached for the same key may come from a class whose largest n (and so its
        // slice) differs within the key's bucket: it applies only if it is a candidate here
        bool fits = false;
        for (const auto &cand : cands) fits = fits || (cand.first == t.threads && cand.second == t.workers);
        if (cached && t.threads > 0 && fits) {
            c.worker_threads = t.threads;
            c.workers = t.workers;
            c.grid = shape_grid(c, sms, false);
        }
        if (report) {
            ClassTuning r = t;
            r.bits = c.bits;
            r.cl = c.cl;
            r.band = c.band;
            r.nmax = c.nmax;
            r.members = (int)c.members.size();
            r.threads = c.worker_threads;
            r.workers = c.workers;
            r.grid = c.grid;
            report->push_back(r);
        }
        if (std::getenv("PIMQAP_TRACE"))
            std::fprintf(stderr, "[pimqap] tuned class bits=%d cl=%d band=%d nmax=%d: %d x %d threads "
                                 "(fixed rule %d x %d: %.3f ms, tuned %.3f ms, %d shapes timed)\n",
                         c.bits, c.cl, c.band, c.nmax, c.workers, c.worker_threads, t.fixed_workers,
                         t.fixed_threads, t.fixed_ms, t.tuned_ms, t.tried);
    }
    return PIMQAP_OK;
}

// One class: instance heads in one pinned image (one copy), tails cleared in one memset,
// queue filled with every active instance's epoch-0 items, largest first.
pimqap_status ClassRun::prepare(const pimqap_instance *insts, const pimqap_params *params,
                                const std::vector<Plan> &plans, const BatchClass &c,
                                const EventLink *ev) {
    cls = c;
    const int m = (int)c.members.size();
    size_t head_total = 0, tail_total = 0, reps_total = 0, perm_total = 0;
    std::vector<size_t> hoff(m), toff(m);
    perm_off.assign(m, 0);
    energy_off.assign(m, 0);
    for (int i = 0; i < m; ++i) {
        const Plan &P = plans[c.members[i]];
        hoff[i] = head_total;
        toff[i] = tail_total;
        head_total += carve_size(P.head);
        tail_total += carve_size(P.tail);
        energy_off[i] = (long long)reps_total;
        reps_total += (size_t)P.T * P.R;
        perm_off[i] = (long long)perm_total;
        perm_total += (size_t)P.n;
    }
    energy_total = reps_total;
    unsigned qcap = 1;
    while (qcap < reps_total + 1) qcap <<= 1;
    const size_t misc = carve_size(sizeof(SolveDev) * m) + 5 * carve_size(8 * (size_t)m) +
                        2 * carve_size(8 * (size_t)qcap) + 8 * carve_size(8) +
                        carve_size(sizeof(BatchResultDev) * m) + carve_size(4 * perm_total) +
                        carve_size(8 * reps_total);
    bytes = head_total + tail_total + misc;
    trace("class: sizes");
    PQ_CUDA(cudaMalloc(&base, bytes));
    trace("class: cudaMalloc");
    PQ_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    PQ_CUDA(cudaMallocHost(&pinned, head_total + 64));
    trace("class: cudaMallocHost");
    for (int i = 0; i < m; ++i) {
        const int k = c.members[i];
        fill_head(&insts[k], &params[k], plans[k], pinned + hoff[i]);
    }
    trace("class: fill heads");
    devs.resize(m);
    beta0s.resize(m);
    ratios.resize(m);
    for (int i = 0; i < m; ++i) {
        const int k = c.members[i];
        beta0s[i] = params[k].beta_internal ? params[k].beta_max : params[k].beta_max * 1.44269504089;
        ratios[i] = params[k].beta_ratio;
        carve_instance(plans[k], base + hoff[i], base + head_total + toff[i], &devs[i]);
        devs[i].goal = params[k].goal;
        devs[i].seed = params[k].seed;
        if (ev) {
            devs[i].ev = *ev;
            devs[i].ev.tag = k;
        }
    }
    PQ_CUDA(cudaMemcpyAsync(base, pinned, head_total, cudaMemcpyHostToDevice, stream));
    PQ_CUDA(cudaMemsetAsync(base + head_total, 0, tail_total + misc, stream));
    for (int i = 0; i < m; ++i) PQ_CUDA(pimqap::launch_setup(devs[i], c.bits, stream));
    trace("class: upload + setup launches");

    char *cur = base + head_total + tail_total;
    d_inst = carve<SolveDev>(cur, m);
    int32_t *d_sym = reinterpret_cast<int32_t *>(carve<int64_t>(cur, m));
    int64_t *d_maxm = carve<int64_t>(cur, m);
    unsigned int *d_finish = reinterpret_cast<unsigned int *>(carve<int64_t>(cur, m));
    long long *d_poff = carve<long long>(cur, m);
    unsigned long long *d_items = carve<unsigned long long>(cur, qcap);
    unsigned long long *d_seq = carve<unsigned long long>(cur, qcap);
    unsigned long long *d_head = carve<unsigned long long>(cur, 1);
    unsigned long long *d_tail = carve<unsigned long long>(cur, 1);
    int32_t *d_active = reinterpret_cast<int32_t *>(carve<int64_t>(cur, 1));
    d_error = reinterpret_cast<int32_t *>(carve<int64_t>(cur, 1));
    d_start = carve<unsigned long long>(cur, 1);
    int32_t *d_shutdown = reinterpret_cast<int32_t *>(carve<int64_t>(cur, 1));
    carve<int64_t>(cur, 2);
    d_results = carve<BatchResultDev>(cur, m);
    d_perms = carve<int32_t>(cur, perm_total);
    d_energies = carve<long long>(cur, reps_total);
    d_energy_off = carve<long long>(cur, m);

    // stop epochs after setup: an instance whose goal is met at mega-iteration 0 never runs
    PQ_CUDA(cudaStreamSynchronize(stream));
    trace("class: setup sync");
    std::vector<int32_t> sym(2 * m, 0);
    std::vector<int64_t> maxm(m);
    std::vector<int32_t> stop0(m);
    for (int i = 0; i < m; ++i) {
        sym[i] = plans[c.members[i]].sym ? 1 : 0;
        maxm[i] = params[c.members[i]].max_megaiters;
        PQ_CUDA(cudaMemcpy(&stop0[i], devs[i].stop_epoch, 4, cudaMemcpyDeviceToHost));
    }
    std::vector<int> order_idx(m);
    for (int i = 0; i < m; ++i) order_idx[i] = i;
    std::stable_sort(order_idx.begin(), order_idx.end(), [&](int a, int b) {
        const Plan &A = plans[c.members[a]], &B = plans[c.members[b]];
        return (double)A.n * A.n * A.T * A.R > (double)B.n * B.n * B.T * B.R;
    });
    std::vector<unsigned long long> items, seq;
    int active = 0;
    for (int i : order_idx) {
        const Plan &P = plans[c.members[i]];
        if (maxm[i] <= 0 || stop0[i] <= 0) continue;
        ++active;
        for (int r = 0; r < P.T * P.R; ++r) {
            items.push_back(((unsigned long long)i << 32) | (unsigned)r);
            seq.push_back(items.size());
        }
    }
    runnable = active;
    const unsigned long long tail = items.size();
    const int32_t shutdown = 1;   // a batch ends when its last instance does
    PQ_CUDA(cudaMemcpyAsync(d_inst, devs.data(), sizeof(SolveDev) * m, cudaMemcpyHostToDevice, stream));
    PQ_CUDA(cudaMemcpyAsync(d_sym, sym.data(), 4 * (size_t)m, cudaMemcpyHostToDevice, stream));
    PQ_CUDA(cudaMemcpyAsync(d_maxm, maxm.data(), 8 * (size_t)m, cudaMemcpyHostToDevice, stream));
    PQ_CUDA(cudaMemcpyAsync(d_poff, perm_off.data(), 8 * (size_t)m, cudaMemcpyHostToDevice, stream));
    PQ_CUDA(cudaMemcpyAsync(d_energy_off, energy_off.data(), 8 * (size_t)m, cudaMemcpyHostToDevice, stream));
    if (!items.empty()) {
        PQ_CUDA(cudaMemcpyAsync(d_items, items.data(), 8 * items.size(), cudaMemcpyHostToDevice, stream));
        PQ_CUDA(cudaMemcpyAsync(d_seq, seq.data(), 8 * seq.size(), cudaMemcpyHostToDevice, stream));
    }
    PQ_CUDA(cudaMemcpyAsync(d_tail, &tail, 8, cudaMemcpyHostToDevice, stream));
    PQ_CUDA(cudaMemcpyAsync(d_active, &active, 4, cudaMemcpyHostToDevice, stream));
    PQ_CUDA(cudaMemcpyAsync(d_shutdown, &shutdown, 4, cudaMemcpyHostToDevice, stream));
    PQ_CUDA(cudaStreamSynchronize(stream));
    trace("class: queue ready");
    d_perm_off = d_poff;

    B = pimqap::BatchDev{};
    B.inst = d_inst; B.sym = d_sym; B.max_megaiters = d_maxm; B.finish_inst = d_finish;
    B.count = m; B.q_items = d_items; B.q_seq = d_seq; B.q_head = d_head; B.q_tail = d_tail;
    B.qmask = qcap - 1; B.active = d_active; B.error = d_error; B.start_ns = d_start;
    B.shutdown = d_shutdown;
    B.serving = 0;
    B.worker_threads = c.worker_threads; B.workers = c.workers; B.slice_bytes = (unsigned)c.slice;
    return PIMQAP_OK;
}

pimqap_status ClassRun::launch() {
    PQ_CUDA(cudaEventCreate(&e0));
    PQ_CUDA(cudaEventCreate(&e1));
    PQ_CUDA(cudaEventRecord(e0, stream));
    if (runnable > 0) PQ_CUDA(pimqap::launch_batch(B, cls.bits, cls.cl, cls.grid, stream));
    PQ_CUDA(pimqap::launch_collect(d_inst, B.count, d_results, d_perms, d_perm_off, d_energies,
                                   d_energy_off, stream));
    PQ_CUDA(cudaEventRecord(e1, stream));
    return PIMQAP_OK;
}

pimqap_status ClassRun::finish(const std::vector<Plan> &plans, pimqap_result *results) {
    PQ_CUDA(cudaStreamSynchronize(stream));
    trace("class: kernel done");
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    const int m = B.count;
    std::vector<pimqap::BatchResultDev> out(m);
    size_t perm_total = 0;
    for (int k : cls.members) perm_total += (size_t)plans[k].n;
    std::vector<int32_t> perms(perm_total);
    std::vector<long long> energies(energy_total);
    int32_t err = 0;
    unsigned long long start_ns = 0;
    PQ_CUDA(cudaMemcpy(&err, d_error, 4, cudaMemcpyDeviceToHost));
    PQ_CUDA(cudaMemcpy(&start_ns, d_start, 8, cudaMemcpyDeviceToHost));
    this->start_ns = start_ns;
    PQ_CUDA(cudaMemcpy(out.data(), d_results, sizeof(pimqap::BatchResultDev) * m, cudaMemcpyDeviceToHost));
    if (perm_total) PQ_CUDA(cudaMemcpy(perms.data(), d_perms, 4 * perm_total, cudaMemcpyDeviceToHost));
    if (energy_total)
        PQ_CUDA(cudaMemcpy(energies.data(), d_energies, 8 * energy_total, cudaMemcpyDeviceToHost));
    if (err) return fail(PIMQAP_ERR_DEVICE, "batch kernel check failed (error word " + std::to_string(err) + ")");
    for (int i = 0; i < m; ++i) {
        const int k = cls.members[i];
        const Plan &P = plans[k];
        const pimqap::BatchResultDev &o = out[i];
        if (o.error) return fail(PIMQAP_ERR_DEVICE, "device check failed in batch instance " + std::to_string(k));
        pimqap_result &R = results[k];
        int32_t *perm_dst = R.best_perm;
        int64_t *energy_dst = R.final_energies;
        std::memset(&R, 0, sizeof(R));
        R.best_perm = perm_dst;
        R.final_energies = energy_dst;
        R.best_energy = std::min<int64_t>(o.best, o.single_best);
        if (perm_dst) std::memcpy(perm_dst, perms.data() + perm_off[i], 4 * (size_t)P.n);
        if (energy_dst) std::memcpy(energy_dst, energies.data() + energy_off[i], 8 * (size_t)P.T * P.R);
        R.target_megaiter = (o.target_epoch == std::numeric_limits<long long>::max()) ? -1 : o.target_epoch;
        R.time_to_target_ms = (R.target_megaiter >= 0 && o.target_ns != ~0ull && o.target_ns >= start_ns)
                                  ? (double)(o.target_ns - start_ns) * 1e-6
                                  : (R.target_megaiter >= 0 ? 0.0 : -1.0);
        R.megaiters_done = o.epoch;
        R.updates = (int64_t)o.epoch * P.spe * P.n * (int64_t)P.T * P.R;
        R.sweeps = R.updates / P.n;
        R.proposals = R.sweeps * ((int64_t)P.n * (P.n - 1) / 2);
        R.accepts = (int64_t)o.accepts;
        R.device_ms = ms;
        R.force_bits = P.bits;
        R.cluster_size = cls.cl;
        R.stopped_by = (o.stop_epoch != pimqap::kNoStop) ? 1 : 0;
        R.h2d_bytes = P.h2d_bytes;
        R.d2h_bytes = (int64_t)(sizeof(pimqap::BatchResultDev) + 4 * (size_t)P.n + 8 * (size_t)P.T * P.R);
        R.beta_max_used = beta0s[i];
        R.beta_ratio_used = ratios[i];
    }
    device_ms = ms;
    trace("class: results");
    return PIMQAP_OK;
}

ClassRun::~ClassRun() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (stream) cudaStreamDestroy(stream);
    if (pinned) cudaFreeHost(pinned);
    if (base) cudaFree(base);
}

}  // namespace detail
}  // namespace pimqap

using namespace pimqap::detail;

extern "C" pimqap_status pimqap_batch_solve(const pimqap_instance *insts, const pimqap_params *params,
                                            int32_t count, pimqap_result *results) {
    return batch_solve(insts, params, count, results, nullptr);
}

namespace pimqap {
namespace detail {

pimqap_status batch_solve(const pimqap_instance *insts, const pimqap_params *params, int32_t count,
                          pimqap_result *results, EventBuffer *ev) {
    if (count < 0 || (count > 0 && (!insts || !params || !results)))
        return fail(PIMQAP_ERR_ARG, "bad batch arguments");
    if (count == 0) return PIMQAP_OK;
    const auto wall0 = std::chrono::steady_clock::now();
    trace("batch: start");
    for (int k = 0; k < count; ++k) {
        pimqap_status st = check_params(&insts[k], &params[k]);
        if (st != PIMQAP_OK) return st;
        if (params[k].active_facilities > 0)
            return fail(PIMQAP_ERR_ARG, "active_facilities is supported by pimqap_solve and solver handles only");
        if (params[k].update_rule != PIMQAP_RULE_SEQUENTIAL)
            return fail(PIMQAP_ERR_ARG, "the one-shot rule is supported by pimqap_solve and solver handles only");
        if (params[k].device != params[0].device)
            return fail(PIMQAP_ERR_ARG, "every batch entry must use the same device");
    }
    int maxsm = 0;
    pimqap_status st = open_device(params[0].device, &maxsm);
    if (st != PIMQAP_OK) return st;
    int sms = 0;
    PQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, params[0].device));
    std::vector<Plan> plans(count);
    std::vector<int64_t> megaiters(count);
    for (int k = 0; k < count; ++k) {
        st = plan_instance(&insts[k], &params[k], (size_t)maxsm, params[k].cluster_size, &plans[k]);
        if (st != PIMQAP_OK) return st;
        megaiters[k] = params[k].max_megaiters;
    }
    trace("batch: plans");
    std::vector<BatchClass> classes = plan_classes(plans, megaiters, sms, maxsm, 0);
    if (autotune_enabled()) {
        st = tune_classes(insts, params, count, plans, classes, sms, maxsm, nullptr);
        if (st != PIMQAP_OK) return st;
    }
    if (std::getenv("PIMQAP_TRACE"))
        for (const auto &c : classes)
            std::fprintf(stderr, "[pimqap] class bits=%d cl=%d band=%d members=%zu work=%.3g grid=%d workers=%d x %d threads slice=%zu\n",
                         c.bits, c.cl, c.band, c.members.size(), c.work, c.grid, c.workers, c.worker_threads, c.slice);
    trace("batch: classes");
    std::vector<std::unique_ptr<ClassRun>> runs;
    for (const auto &c : classes) {
        runs.emplace_back(new ClassRun());
        st = runs.back()->prepare(insts, params, plans, c, ev ? &ev->link : nullptr);
        if (st != PIMQAP_OK) return st;
    }
    for (auto &r : runs) {   // all classes run concurrently, each on its own stream
        st = r->launch();
        if (st != PIMQAP_OK) return st;
    }
    unsigned long long t0 = ~0ull;
    for (auto &r : runs) {
        st = r->finish(plans, results);
        if (st != PIMQAP_OK) return st;
        if (r->runnable > 0) t0 = std::min(t0, r->start_ns);
    }
    if (ev) {
        st = ev->drain(runs.front()->stream, t0 == ~0ull ? 0ull : t0, false);
        if (st != PIMQAP_OK) return st;
    }
    runs.clear();
    trace("batch: released");
    const double el = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall0).count();
    for (int k = 0; k < count; ++k) results[k].wall_ms = el;
    return PIMQAP_OK;
}

}  // namespace detail
}  // namespace pimqap

extern "C" pimqap_status pimqap_batch_tune(const pimqap_instance *insts, const pimqap_params *params,
                                           int32_t count, pimqap_class_tuning *out, int32_t capacity,
                                           int32_t *class_count) {
    if (count < 1 || !insts || !params || !class_count || capacity < 0 || (capacity > 0 && !out))
        return fail(PIMQAP_ERR_ARG, "bad tuning arguments");
    *class_count = 0;
    for (int k = 0; k < count; ++k) {
        pimqap_status st = check_params(&insts[k], &params[k]);
        if (st != PIMQAP_OK) return st;
        if (params[k].active_facilities > 0 || params[k].update_rule != PIMQAP_RULE_SEQUENTIAL ||
            params[k].device != params[0].device)
            return fail(PIMQAP_ERR_ARG, "batch entries: sequential rule, no active_facilities, one device");
    }
    int maxsm = 0;
    pimqap_status st = open_device(params[0].device, &maxsm);
    if (st != PIMQAP_OK) return st;
    int sms = 0;
    PQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, params[0].device));
    std::vector<Plan> plans(count);
    std::vector<int64_t> megaiters(count);
    for (int k = 0; k < count; ++k) {
        st = plan_instance(&insts[k], &params[k], (size_t)maxsm, params[k].cluster_size, &plans[k]);
        if (st != PIMQAP_OK) return st;
        megaiters[k] = params[k].max_megaiters;
    }
    std::vector<BatchClass> classes = plan_classes(plans, megaiters, sms, maxsm, 0);
    std::vector<ClassTuning> report;
    if (autotune_enabled()) {
        st = tune_classes(insts, params, count, plans, classes, sms, maxsm, &report);
        if (st != PIMQAP_OK) return st;
    } else {
        for (const auto &c : classes) {
            ClassTuning r{};
            r.bits = c.bits; r.cl = c.cl; r.band = c.band; r.nmax = c.nmax;
            r.members = (int)c.members.size(); r.threads = c.worker_threads; r.workers = c.workers;
            r.grid = c.grid; r.fixed_threads = c.worker_threads; r.fixed_workers = c.workers;
            report.push_back(r);
        }
    }
    *class_count = (int32_t)report.size();
    for (int i = 0; i < (int)report.size() && i < capacity; ++i) {
        const ClassTuning &r = report[i];
        pimqap_class_tuning &o = out[i];
        std::memset(&o, 0, sizeof(o));
        o.force_bits = r.bits; o.cluster_size = r.cl; o.band = r.band; o.n_max = r.nmax;
        o.members = r.members; o.threads = r.threads; o.workers = r.workers; o.grid = r.grid;
        o.fixed_threads = r.fixed_threads; o.fixed_workers = r.fixed_workers; o.tried = r.tried;
        o.fixed_ms = r.fixed_ms; o.tuned_ms = r.tuned_ms;
    }
    return PIMQAP_OK;
}

namespace {

uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

}  // namespace

// autoSelectParameters (CPU_PIM.cpp:366-476).  The reference runs the trials one after another
// with fresh random_device seeds; here trial (k, t) is seeded with splitmix64(seed + 5k + t + 1)
// and all 160 trials run in one batched launch.  The averaging order and the selection rule are
// the reference's, in the same double arithmetic.  Because the reference's trials run in order
// and its best energy carries over between them, the first trial (in that order) whose tracked
// best reaches the goal ends automatic mode (:419-422); the trials after it are ignored.
// ------------------------------------------------------------------ asynchronous batches

// A batch solved on its own host thread: the instances and parameters are copied at submit,
// the caller's result array (and its best_perm / final_energies buffers) is written when the
// batch finishes and must stay alive until pimqap_batch_poll / pimqap_batch_wait reports it.
struct pimqap_batch {
    std::vector<std::vector<int32_t>> flows, dists;
    std::vector<pimqap_instance> insts;
    std::vector<pimqap_params> params;
    pimqap_result *results = nullptr;
    std::thread worker;
    std::atomic<int> done{0};
    pimqap_status status = PIMQAP_OK;
    std::string error;
};

extern "C" pimqap_status pimqap_batch_submit(const pimqap_instance *insts, const pimqap_params *params,
                                             int32_t count, pimqap_result *results, pimqap_batch **out) {
    if (!out) return fail(PIMQAP_ERR_ARG, "null batch handle");
    *out = nullptr;
    if (!insts || !params || !results || count < 1) return fail(PIMQAP_ERR_ARG, "empty batch");
    std::unique_ptr<pimqap_batch> b(new pimqap_batch());
    b->flows.resize(count);
    b->dists.resize(count);
    b->insts.resize(count);
    for (int k = 0; k < count; ++k) {
        const int n = insts[k].n;
        if (n < 1 || n > PIMQAP_MAX_N || !insts[k].flow || !insts[k].dist)
            return fail(PIMQAP_ERR_ARG, "instance " + std::to_string(k) + " is malformed");
        b->flows[k].assign(insts[k].flow, insts[k].flow + (size_t)n * n);
        b->dists[k].assign(insts[k].dist, insts[k].dist + (size_t)n * n);
        b->insts[k] = pimqap_instance{n, b->flows[k].data(), b->dists[k].data()};
    }
    b->params.assign(params, params + count);
    b->results = results;
    pimqap_batch *raw = b.get();
    raw->worker = std::thread([raw, count] {
        raw->status = pimqap_batch_solve(raw->insts.data(), raw->params.data(), count, raw->results);
        if (raw->status != PIMQAP_OK) raw->error = pimqap_last_error();
        raw->done.store(1, std::memory_order_release);
    });
    *out = b.release();
    return PIMQAP_OK;
}

extern "C" pimqap_status pimqap_batch_poll(pimqap_batch *b) {
    if (!b) return fail(PIMQAP_ERR_ARG, "null batch handle");
    if (!b->done.load(std::memory_order_acquire)) return PIMQAP_ERR_NOT_READY;
    if (b->worker.joinable()) b->worker.join();
    if (b->status != PIMQAP_OK) return fail(b->status, b->error);
    return PIMQAP_OK;
}

extern "C" pimqap_status pimqap_batch_wait(pimqap_batch *b, double timeout_s) {
    if (!b) return fail(PIMQAP_ERR_ARG, "null batch handle");
    const auto t0 = std::chrono::steady_clock::now();
    while (!b->done.load(std::memory_order_acquire)) {
        if (timeout_s >= 0 &&
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() >= timeout_s)
            return PIMQAP_ERR_NOT_READY;
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
    return pimqap_batch_poll(b);
}

extern "C" void pimqap_batch_release(pimqap_batch *b) {
    if (!b) return;
    if (b->worker.joinable()) b->worker.join();
    delete b;
}

extern "C" pimqap_status pimqap_auto_beta_report(const pimqap_instance *inst, const pimqap_params *params,
                                                 pimqap_auto_report *rep) {
    if (!inst || !params || !rep) return fail(PIMQAP_ERR_ARG, "null argument");
    pimqap_status st = check_params(inst, params);
    if (st != PIMQAP_OK) return st;
    if (params->active_facilities > 0)
        return fail(PIMQAP_ERR_ARG, "automatic mode with active_facilities is not supported: give beta_max");
    if (params->update_rule != PIMQAP_RULE_SEQUENTIAL)
        return fail(PIMQAP_ERR_ARG, "automatic mode with the one-shot rule is not supported: give beta_max");
    constexpr double kMinBetaToTry = -30, kBetaStep = 1;     // :366-370
    constexpr int kTrials = PIMQAP_AUTO_TRIALS, kSteps = PIMQAP_AUTO_STEPS, kMegaiters = 10;  // :368, :371, :391
    const int T = params->groups, R = params->replicas, n = inst->n;
    std::vector<pimqap_instance> insts(kSteps * kTrials, *inst);
    std::vector<pimqap_params> ps(kSteps * kTrials, *params);
    for (int i = 0; i < kSteps; ++i)
        for (int t = 0; t < kTrials; ++t) {
            pimqap_params &p = ps[i * kTrials + t];
            p.auto_beta = 0;
            p.beta_internal = 1;
            p.beta_max = std::exp2(kMinBetaToTry + i * kBetaStep);   // :396-397
            p.beta_ratio = 1.0;                                       // :389
            p.max_megaiters = kMegaiters;
            p.seed = splitmix64(params->seed + (uint64_t)(i * kTrials + t) + 1);
            p.timeout_s = 0;
            p.goal_print = 0;
            p.event_capacity = 0;
        }
    std::vector<pimqap_result> rs(ps.size());
    std::vector<std::vector<int64_t>> energies(ps.size(), std::vector<int64_t>((size_t)T * R));
    std::vector<std::vector<int32_t>> perms(ps.size(), std::vector<int32_t>(n));
    for (size_t k = 0; k < rs.size(); ++k) {
        std::memset(&rs[k], 0, sizeof(pimqap_result));
        rs[k].final_energies = energies[k].data();
        rs[k].best_perm = perms[k].data();
    }
    // Group-best events of every trial: the tracked bests (mega-iterations 0-9) decide the goal
    // and give the "Best Energy Found" lines printed during automatic mode.
    EventBuffer ev;
    {
        int maxsm = 0;
        st = open_device(params->device, &maxsm);
        if (st != PIMQAP_OK) return st;
        const unsigned cap = (unsigned)std::min<size_t>((size_t)1 << 22, (size_t)ps.size() * T * R * (kMegaiters + 1));
        st = ev.allocate(cap, 0, n, 0, 0);
        if (st != PIMQAP_OK) return st;
        PQ_CUDA(cudaStreamSynchronize(0));
    }
    st = batch_solve(insts.data(), ps.data(), (int32_t)ps.size(), rs.data(), &ev);
    if (st != PIMQAP_OK) return st;
    if (ev.dropped) return fail(PIMQAP_ERR_ARG, "automatic mode: event log overflow");

    const int ntrial = kSteps * kTrials;
    for (int k = 0; k < ntrial; ++k) rep->trial_best[k] = PIMQAP_NO_BEST;
    for (const pimqap_event &e : ev.events)
        if (e.kind == PIMQAP_EVENT_GROUP_BEST && e.megaiter < kMegaiters)
            rep->trial_best[e.trial] = std::min<int64_t>(rep->trial_best[e.trial], e.energy);
    int goal_trial = -1;
    for (int k = 0; k < ntrial && goal_trial < 0; ++k)
        if (rep->trial_best[k] <= params->goal) goal_trial = k;
    const int used = goal_trial >= 0 ? goal_trial + 1 : ntrial;

    double sums[kSteps] = {0};
    const double denom = static_cast<double>(kTrials) * T * R;                    // :412
    for (int i = 0; i < kSteps; ++i)
        for (int t = 0; t < kTrials; ++t)
            for (int g = 0; g < T; ++g)
                for (int l = 0; l < R; ++l)
                    sums[i] += (double)energies[i * kTrials + t][(size_t)g * R + l] / denom;
    size_t arg = 0;
    for (int k = 1; k < used; ++k)
        if (rs[k].best_energy < rs[arg].best_energy) arg = k;
    rep->best_energy = rs[arg].best_energy;
    if (rep->best_perm) std::memcpy(rep->best_perm, perms[arg].data(), 4 * (size_t)n);
    std::memcpy(rep->avg_energy, sums, sizeof(sums));
    rep->goal_trial = goal_trial;
    rep->device_ms = rs[0].device_ms;
    rep->event_count = 0;
    rep->events_dropped = 0;
    for (const pimqap_event &e : ev.events) {
        if (e.kind != PIMQAP_EVENT_GROUP_BEST || e.megaiter >= kMegaiters || e.trial >= used) continue;
        if (rep->events && rep->event_count < rep->event_capacity) rep->events[rep->event_count++] = e;
        else ++rep->events_dropped;
    }
    rep->min_beta = rep->max_beta = 0;
    rep->min_beta_printed = 0;
    if (goal_trial >= 0) {                   // :419-422: beta0 stays at the step's beta
        rep->steps_printed = goal_trial / kTrials;
        rep->beta0_internal = std::exp2(kMinBetaToTry + (goal_trial / kTrials) * kBetaStep);
        rep->delta_beta = 1.0;
        return PIMQAP_OK;
    }
    rep->steps_printed = kSteps;
    const int i = kSteps - 1;                                                       // :434
    double minE = 1e30, maxE = -1e30;
    int minEIndex = 0;
    for (int j = 0; j < i; j++) {                                                   // :438-446
        if (sums[j] < minE) {
            minE = sums[j];
            minEIndex = j;
        }
        if (j == 0) maxE = sums[j];
    }
    double minBeta = 0, maxBeta = 0;
    const double higher = params->auto_higher, lower = params->auto_lower;
    for (int j = 0; j < i; j++) {                                                   // :447-473
        if (minBeta == 0 && ((j == (minEIndex - 1) && (j >= 1)) || (sums[j] < (maxE - minE) * higher + minE))) {
            minBeta = std::exp2(kMinBetaToTry + (j)*kBetaStep);
            rep->min_beta_printed = 1;
        }
        if (j == i - 1 || (minBeta != 0 && (j == minEIndex || (sums[j] < (maxE - minE) * lower + minE)))) {
            if (minBeta == 0) minBeta = std::exp2(kMinBetaToTry + 0 * kBetaStep);
            maxBeta = std::exp2(kMinBetaToTry + (j + 2) * kBetaStep);
            rep->min_beta = minBeta;
            rep->max_beta = maxBeta;
            rep->beta0_internal = maxBeta;
            rep->delta_beta = std::pow(maxBeta / minBeta, 1.0 / R);
            return PIMQAP_OK;
        }
    }
    return fail(PIMQAP_ERR_ARG, "automatic beta selection found no range");
}

extern "C" pimqap_status pimqap_auto_beta(const pimqap_instance *inst, const pimqap_params *params,
                                          double *beta0_internal, double *delta_beta, double *avg_energy,
                                          int64_t *best_energy, int32_t *best_perm) {
    if (!beta0_internal || !delta_beta) return fail(PIMQAP_ERR_ARG, "null argument");
    std::unique_ptr<pimqap_auto_report> rep(new pimqap_auto_report());
    std::memset(rep.get(), 0, sizeof(pimqap_auto_report));
    rep->best_perm = best_perm;
    pimqap_status st = pimqap_auto_beta_report(inst, params, rep.get());
    if (st != PIMQAP_OK) return st;
    *beta0_internal = rep->beta0_internal;
    *delta_beta = rep->delta_beta;
    if (avg_energy) std::memcpy(avg_energy, rep->avg_energy, sizeof(rep->avg_energy));
    if (best_energy) *best_energy = rep->best_energy;
    return PIMQAP_OK;
}
