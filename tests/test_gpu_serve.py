"""Serving: continuous batching with resident launches (GPU).

Requests submitted while others run are admitted as slots and device memory free up; each
result must equal pimqap_solve of the same request alone.  A host-side heartbeat stall must
make the device workers' idle waits run out and stop them with an error status.
"""
import time

import numpy as np
import pytest

import instances

pytestmark = pytest.mark.gpu


def same(a, b):
    keys = ("best_energy", "megaiters_done", "updates", "sweeps", "proposals", "accepts", "target_megaiter",
            "stopped_by")
    return all(a[k] == b[k] for k in keys) and np.array_equal(a["best_perm"], b["best_perm"]) \
        and np.array_equal(a["final_energies"], b["final_energies"])


def requests(gpu, count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.integers(8, 200))
        if k % 4 == 3:
            inst = instances.Instance(n, rng.integers(0, 2_000_000, (n, n)), rng.integers(0, 5000, (n, n)))
            b = 1e-9
        else:
            inst = instances.uniform(n, seed * 100 + k)
            b = 0.02
        p = gpu.default_params(replicas=int(rng.integers(2, 12)), groups=1 + k % 2,
                               sweeps_per_exchange=1 + k % 3, beta_max=b, beta_ratio=1.4,
                               seed=seed + k, max_megaiters=int(rng.integers(2, 9)))
        out.append((inst, p))
    return out


def test_served_results_equal_solo_solves(gpu):
    reqs = requests(gpu, 14, 3)
    with gpu.Server() as srv:
        first = [srv.submit(i.F, i.D, p) for i, p in reqs[:7]]
        time.sleep(0.05)                    # the rest arrive while the first are on the GPU
        second = [srv.submit(i.F, i.D, p) for i, p in reqs[7:]]
        st0 = srv.stats()
        assert st0["error_word"] == 0, st0
        got = [srv.wait(t, 120.0) for t in first + second]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["error_word"] == 0, st
    for (inst, p), r in zip(reqs, got):
        assert same(r, gpu.solve(inst.F, inst.D, p)), inst.n
        assert r["latency_ms"] >= r["admit_ms"] >= 0


def test_memory_budget_gates_admission(gpu):
    reqs = requests(gpu, 8, 5)
    sizes = []
    with gpu.Server(memory_budget=24 << 20, slots_per_class=4) as srv:
        tickets = [srv.submit(i.F, i.D, p) for i, p in reqs]
        peak_pending = srv.stats()["pending"]
        got = [srv.wait(t, 120.0) for t in tickets]
        sizes.append(srv.stats()["memory_budget"])
        big = instances.grid256(9)
        p = gpu.default_params(replicas=64, groups=8, max_megaiters=1)
        with pytest.raises(gpu.PimqapError) as e:
            srv.submit(big.F, big.D, p)
        assert e.value.status == 7           # never fits the budget
    assert peak_pending >= 0
    for (inst, p), r in zip(reqs, got):
        assert same(r, gpu.solve(inst.F, inst.D, p))


def test_heartbeat_stall_stops_device_workers(gpu):
    inst = instances.uniform(20, 11)
    p = gpu.default_params(replicas=4, groups=1, max_megaiters=3, beta_max=0.02)
    srv = gpu.Server(heartbeat_timeout=0.5)
    try:
        t = srv.submit(inst.F, inst.D, p)
        srv.wait(t, 60.0)
        srv.stall_heartbeat(True)
        deadline = time.time() + 20
        while time.time() < deadline and srv.stats()["error_word"] == 0:
            time.sleep(0.1)
        assert srv.stats()["error_word"] & 8      # host lost: the bounded idle waits ran out
        with pytest.raises(gpu.PimqapError) as e:
            srv.submit(inst.F, inst.D, p)
        assert e.value.status == 6
    finally:
        srv.close()                               # returns: the workers have already stopped


def test_requests_outside_the_sample_still_find_a_launch(gpu):
    """A server tuned on a sample of small int32 instances still serves a large int64 one
    (classes for the uncovered shapes are added at creation)."""
    small = instances.uniform(24, 5)
    ps = gpu.default_params(replicas=4, groups=1, beta_max=0.02, beta_ratio=1.3, max_megaiters=3)
    n = 240
    rng = np.random.default_rng(11)
    big = instances.Instance(n, rng.integers(0, 30_000_000, (n, n)), rng.integers(0, 100, (n, n)))
    pb = gpu.default_params(replicas=3, groups=1, beta_max=1e-9, beta_ratio=1.3, seed=4, max_megaiters=2)
    with gpu.Server(sample=[(small.F, small.D, ps)]) as srv:
        t = srv.submit(big.F, big.D, pb)
        r = srv.wait(t, 120.0)
        assert srv.stats()["error_word"] == 0
    solo = gpu.solve(big.F, big.D, pb)
    assert r["force_bits"] == 64 and same(r, solo)


def test_destroy_abandons_running_requests_promptly(gpu):
    """Closing the server with long requests still running stops the resident launches at
    once instead of running the requests to the end."""
    inst = instances.uniform(96, 12)
    p = gpu.default_params(replicas=16, groups=2, beta_max=0.02, beta_ratio=1.3, max_megaiters=10 ** 7)
    srv = gpu.Server()
    for k in range(6):
        p.seed = k + 1
        srv.submit(inst.F, inst.D, p)
    time.sleep(0.5)
    st = srv.stats()
    assert st["admitted"] >= 1 and st["completed"] == 0 and st["error_word"] == 0, st
    t0 = time.perf_counter()
    srv.close()
    assert time.perf_counter() - t0 < 10.0
    r = gpu.solve(inst.F, inst.D, gpu.default_params(replicas=4, groups=1, max_megaiters=3))
    assert r["megaiters_done"] == 3      # the device is usable afterwards
