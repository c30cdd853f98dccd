"""pimqap_solve_static: the solve for callers that cannot allocate device memory.

A program whose device memory is claimed by another allocator, or that may not take the CUDA
allocator's locks or latency while it solves, calls pimqap_solve_static.  It runs the same
kernels as pimqap_solve, but on a fixed 8 MiB device array that the library reserves when it
is loaded, so the call allocates nothing.  These tests call it through the C ABI and check it
against pimqap_solve: results must be identical (integer costs, permutations and counters are
exact; the tolerance is zero, as in every parity test here), on two calls in a row, since
every call reuses - and must first clear - the same array.
"""
import numpy as np
import pytest

import instances

pytestmark = pytest.mark.gpu

CASES = [
    # (instance, params)
    (lambda: instances.uniform(32, 301), dict(replicas=8, groups=2, sweeps_per_exchange=1,
                                              beta_max=0.05, beta_ratio=1.3, max_megaiters=30)),
    (lambda: instances.grid256(302), dict(replicas=4, groups=1, sweeps_per_exchange=2,
                                          beta_max=0.002, beta_ratio=1.5, max_megaiters=3)),
    (lambda: instances.heavy(90, 303), dict(replicas=6, groups=2, sweeps_per_exchange=4,
                                            beta_max=1e-5, beta_ratio=1.6, max_megaiters=5)),
]


def same(a, b):
    keys = ("best_energy", "megaiters_done", "updates", "sweeps", "proposals", "accepts", "target_megaiter",
            "stopped_by")
    return all(a[k] == b[k] for k in keys) and np.array_equal(a["best_perm"], b["best_perm"])


@pytest.mark.parametrize("idx", range(len(CASES)))
def test_static_solve_matches_pimqap_solve_twice(gpu, idx):
    make, kw = CASES[idx]
    inst = make()
    p = gpu.default_params(seed=17 + idx, **kw)
    ref = gpu.solve(inst.F, inst.D, p)
    for _ in range(2):                      # the second call must not see the first's state
        got = gpu.solve_static(inst.F, inst.D, p)
        assert same(got, ref), (got, ref)


def test_static_solve_goal_stop_matches(gpu):
    inst = instances.uniform(24, 311)
    base = dict(replicas=6, groups=2, sweeps_per_exchange=1, beta_max=0.05, beta_ratio=1.3,
                max_megaiters=60, megaiters_per_launch=4)
    probe = gpu.solve(inst.F, inst.D, gpu.default_params(seed=5, **base))
    p = gpu.default_params(seed=5, goal=probe["best_energy"] + 800, **base)
    ref = gpu.solve(inst.F, inst.D, p)
    assert ref["stopped_by"] == 1
    for _ in range(2):
        assert same(gpu.solve_static(inst.F, inst.D, p), ref)


def test_static_solve_timeout_stop_matches(gpu):
    """The -s stop (CPU_PIM.cpp:350-357) on this entry point: stopped_by = 2 only when
    mega-iterations were left when the time ran out, as pimqap_solve reports it."""
    import time
    inst = instances.uniform(48, 314)
    base = dict(replicas=8, groups=4, sweeps_per_exchange=4, beta_max=0.05, beta_ratio=1.3,
                megaiters_per_launch=8, seed=9)
    p = gpu.default_params(timeout_s=0.3, max_megaiters=2 ** 40, **base)
    for _ in range(2):
        t0 = time.perf_counter()
        got = gpu.solve_static(inst.F, inst.D, p)
        assert time.perf_counter() - t0 < 0.3 + 10.0
        assert got["stopped_by"] == 2 and 0 < got["megaiters_done"] < p.max_megaiters
        perm = got["best_perm"]
        assert int((inst.D.astype(np.int64) * inst.F[np.ix_(perm, perm)]).sum()) == got["best_energy"]
    assert gpu.solve(inst.F, inst.D, p)["stopped_by"] == 2
    # every mega-iteration ran before the time ran out: no timeout stop, on both entry points
    q = gpu.default_params(timeout_s=600.0, max_megaiters=6, **base)
    ref = gpu.solve(inst.F, inst.D, q)
    assert ref["stopped_by"] == 0
    assert same(gpu.solve_static(inst.F, inst.D, q), ref)


def test_static_solve_leaves_free_device_memory_unchanged(gpu):
    """The entry point's defining claim: a call allocates no device memory.  Free device memory
    is read after warm-up calls of every shape used below (the first launch of a kernel may load
    its module) and after the blocks that solver handles keep are released."""
    import torch
    shapes = [(instances.uniform(32, 321), dict(replicas=8, groups=2, max_megaiters=6, beta_max=0.05)),
              (instances.heavy(90, 322), dict(replicas=6, groups=2, max_megaiters=3, beta_max=1e-5)),
              (instances.grid256(323), dict(replicas=4, groups=1, max_megaiters=2, beta_max=0.002))]
    for inst, kw in shapes:
        gpu.solve_static(inst.F, inst.D, gpu.default_params(seed=1, **kw))
    gpu.release_kept_memory()
    torch.cuda.synchronize(0)
    free0, _ = torch.cuda.mem_get_info(0)
    for rep in range(2):
        for inst, kw in shapes:
            gpu.solve_static(inst.F, inst.D, gpu.default_params(seed=2 + rep, **kw))
    torch.cuda.synchronize(0)
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"


def test_static_solve_rejects_oversized(gpu):
    inst = instances.grid256(312)
    p = gpu.default_params(replicas=64, groups=1, max_megaiters=1)   # 64 x 256 KiB of force matrices
    with pytest.raises(gpu.PimqapError) as e:
        gpu.solve_static(inst.F, inst.D, p)
    assert e.value.status == 1 and "static scratch" in str(e.value)
    # a rejected call leaves the entry point usable
    small = instances.uniform(16, 313)
    q = gpu.default_params(replicas=4, groups=1, max_megaiters=5, beta_max=0.05, seed=2)
    assert same(gpu.solve_static(small.F, small.D, q), gpu.solve(small.F, small.D, q))
