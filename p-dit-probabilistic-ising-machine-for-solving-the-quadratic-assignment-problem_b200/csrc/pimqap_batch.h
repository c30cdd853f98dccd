// pimqap_batch.h - classes of a batch (the autotuner's choices) and the runtime of one
// persistent class launch.  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "pimqap.h"
#include "pimqap_internal.h"
#include "pimqap_plan.h"
#include "pimqap_events.h"

namespace pimqap {
namespace detail {

// One persistent launch: instances of one force-matrix width and cluster size (and, for
// single-CTA replicas, one band of n), with the worker shape and grid picked for them.
struct BatchClass {
    int bits = 32, cl = 1, band = 0;
    int nmax = 0;                 // largest n among the members
    std::vector<int> members;     // indices into the batch
    double work = 0;              // estimated cost (relative)
    int worker_threads = 128;     // threads of one replica worker
    int workers = 1;              // workers per CTA
    size_t slice = 0;             // shared memory per worker
    int grid = 1;                 // CTAs of the launch
};

// Relative cost of an instance: updates x (candidates + expected force-update share).
double instance_work(const Plan &P, int64_t megaiters);

// The fixed rules: partitions plans into classes and picks worker shapes from the n range and
// the occupancy of each shape (tune_classes then measures the alternatives).
std::vector<BatchClass> plan_classes(const std::vector<Plan> &plans, const std::vector<int64_t> &megaiters,
                                     int sms, int maxsm, int force_cluster);

// What the autotuner measured for a class shape (device time of one mega-iteration of the
// class's instances under the fixed rules' worker shape and under the fastest one).
struct ClassTuning {
    int bits = 0, cl = 0, band = 0, nmax = 0, members = 0;
    int threads = 0, workers = 0, grid = 0;   // the shape in use
    int fixed_threads = 0, fixed_workers = 0; // the fixed rules' shape
    int tried = 0;                            // shapes timed (0: from the cache or nothing to choose)
    double fixed_ms = 0, tuned_ms = 0, work = 0;
};

// PIMQAP_AUTOTUNE=0 in the environment turns the autotuner off (the fixed rules' shapes).
bool autotune_enabled();

// The autotuner: for every class whose shape is not cached yet, times one mega-iteration of its
// members under each candidate worker shape and keeps the fastest (shapes never change results);
// applies the cached choice to every class.  `report` (may be null) receives one entry per class.
// one_per_sm: shapes are timed with one CTA (cluster) per SM, as the serving launches run them.
pimqap_status tune_classes(const pimqap_instance *insts, const pimqap_params *params, int32_t count,
                           const std::vector<Plan> &plans, std::vector<BatchClass> &classes, int sms,
                           int maxsm, std::vector<ClassTuning> *report, bool one_per_sm = false);

// Device state and stream of one class launch.
struct ClassRun {
    BatchClass cls;
    pimqap::BatchDev B{};
    std::vector<SolveDev> devs;
    std::vector<long long> perm_off, energy_off;
    std::vector<double> beta0s, ratios;   // beta0 (internal units) and deltaBeta per member
    char *base = nullptr;
    char *pinned = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    SolveDev *d_inst = nullptr;
    pimqap::BatchResultDev *d_results = nullptr;
    int32_t *d_perms = nullptr;
    long long *d_perm_off = nullptr;
    long long *d_energies = nullptr, *d_energy_off = nullptr;
    size_t energy_total = 0;
    int32_t *d_error = nullptr;
    unsigned long long *d_start = nullptr;
    int runnable = 0;
    double device_ms = 0;
    unsigned long long start_ns = 0;   // %globaltimer when the launch started

    // `ev` (may be null): the event log every member appends to, tagged with its batch index.
    pimqap_status prepare(const pimqap_instance *insts, const pimqap_params *params,
                          const std::vector<Plan> &plans, const BatchClass &c,
                          const EventLink *ev = nullptr);
    pimqap_status launch();
    pimqap_status finish(const std::vector<Plan> &plans, pimqap_result *results);
    ~ClassRun();
};

// pimqap_batch_solve with an optional event log shared by all members (tag = batch index);
// the log is drained (times from the earliest class start) before this returns.
pimqap_status batch_solve(const pimqap_instance *insts, const pimqap_params *params, int32_t count,
                          pimqap_result *results, EventBuffer *ev);

}  // namespace detail
}  // namespace pimqap
