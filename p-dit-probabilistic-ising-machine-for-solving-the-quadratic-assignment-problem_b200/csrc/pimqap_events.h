// pimqap_events.h - the device event log behind the reference's progress output ("Best Energy
// Found" lines, sweep<t>.txt, goal-print lines) and its host-side drain.  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "pimqap.h"
#include "pimqap_internal.h"

namespace pimqap {
namespace detail {

// One device log: a counter pair, `cap` EventDev records and `pcap` permutations of n entries.
// The kernels append; drain() copies what was appended since the last drain, puts it in the
// reference's order and (optionally) rewinds the device log for the next run call.
struct EventBuffer {
    char *mem = nullptr;
    EventLink link{};
    int n = 0;
    std::vector<pimqap_event> events;   // drained, in the reference's order per drain
    std::vector<int32_t> perms;         // [kept][n], indexed by pimqap_event::perm_index
    int64_t dropped = 0;

    pimqap_status allocate(unsigned cap, unsigned pcap, int n_, int64_t goal_print, cudaStream_t q);
    // Copies the new records (stream q, synchronous), times them from t0_ns (%globaltimer),
    // sorts them by (tag, mega-iteration, tracking before sweeps, group, replica, append order).
    pimqap_status drain(cudaStream_t q, unsigned long long t0_ns, bool rewind);
    EventBuffer() = default;
    EventBuffer(const EventBuffer &) = delete;
    EventBuffer &operator=(const EventBuffer &) = delete;
    ~EventBuffer();
};

}  // namespace detail
}  // namespace pimqap
