// pimqap_events.cpp - allocation and drain of the device event log.
#include "pimqap_events.h"

#include <algorithm>
#include <numeric>
#include <string>

#include "pimqap_plan.h"

namespace pimqap {
namespace detail {

pimqap_status EventBuffer::allocate(unsigned cap, unsigned pcap, int n_, int64_t goal_print,
                                    cudaStream_t q) {
    n = n_;
    const size_t bytes = 256 + sizeof(EventDev) * (size_t)cap + 4 * (size_t)pcap * (size_t)n;
    PQ_CUDA(cudaMalloc(&mem, bytes));
    PQ_CUDA(cudaMemsetAsync(mem, 0, 256, q));
    link = EventLink{};
    link.count = reinterpret_cast<unsigned int *>(mem);
    link.log = reinterpret_cast<EventDev *>(mem + 256);
    link.perm = pcap ? reinterpret_cast<int32_t *>(mem + 256 + sizeof(EventDev) * (size_t)cap) : nullptr;
    link.cap = cap;
    link.pcap = pcap;
    link.goal_print = goal_print;
    return PIMQAP_OK;
}

pimqap_status EventBuffer::drain(cudaStream_t q, unsigned long long t0_ns, bool rewind) {
    if (!mem) return PIMQAP_OK;
    unsigned cnt[2] = {0, 0};
    PQ_CUDA(cudaMemcpyAsync(cnt, link.count, 8, cudaMemcpyDeviceToHost, q));
    PQ_CUDA(cudaStreamSynchronize(q));
    const unsigned m = std::min(cnt[0], link.cap);
    const unsigned pm = std::min(cnt[1], link.pcap);
    std::vector<EventDev> raw(m);
    if (m) PQ_CUDA(cudaMemcpyAsync(raw.data(), link.log, sizeof(EventDev) * m, cudaMemcpyDeviceToHost, q));
    const size_t pbase = perms.size() / (n > 0 ? (size_t)n : 1);
    if (pm) {
        perms.resize(perms.size() + (size_t)pm * n);
        PQ_CUDA(cudaMemcpyAsync(perms.data() + pbase * n, link.perm, 4 * (size_t)pm * n,
                                cudaMemcpyDeviceToHost, q));
    }
    if (rewind && (cnt[0] || cnt[1])) PQ_CUDA(cudaMemsetAsync(link.count, 0, 8, q));
    PQ_CUDA(cudaStreamSynchronize(q));
    dropped += (int64_t)(cnt[0] - m);
    std::vector<unsigned> idx(m);
    std::iota(idx.begin(), idx.end(), 0u);
    auto key_less = [&](unsigned a, unsigned b) {
        const EventDev &x = raw[a], &y = raw[b];
        if (x.tag != y.tag) return x.tag < y.tag;
        if (x.megaiter != y.megaiter) return x.megaiter < y.megaiter;
        const int kx = x.kind_slot == -1 ? 0 : 1, ky = y.kind_slot == -1 ? 0 : 1;
        if (kx != ky) return kx < ky;
        if (x.group != y.group) return x.group < y.group;
        if (x.replica != y.replica) return x.replica < y.replica;
        return a < b;
    };
    std::sort(idx.begin(), idx.end(), key_less);
    events.reserve(events.size() + m);
    for (unsigned k : idx) {
        const EventDev &x = raw[k];
        pimqap_event e{};
        e.megaiter = x.megaiter;
        e.energy = x.energy;
        e.time_ms = x.ns >= t0_ns ? (double)(x.ns - t0_ns) * 1e-6 : 0.0;
        e.kind = x.kind_slot == -1 ? PIMQAP_EVENT_GROUP_BEST : PIMQAP_EVENT_GOAL_PRINT;
        e.group = x.group;
        e.replica = x.replica;
        e.perm_index = (x.kind_slot >= 0 && (unsigned)x.kind_slot < pm) ? (int32_t)(pbase + x.kind_slot) : -1;
        e.trial = x.tag;
        events.push_back(e);
    }
    return PIMQAP_OK;
}

EventBuffer::~EventBuffer() {
    if (mem) cudaFree(mem);
}

}  // namespace detail
}  // namespace pimqap
