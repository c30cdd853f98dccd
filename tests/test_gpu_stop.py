"""The timeout stop of the reference (-s, CPU_PIM.cpp:350-357; params.timeout_s) on the GPU:
a run with unlimited mega-iterations ends once the time is up, reports stopped_by = 2 and
leaves a consistent state (the reported best permutation has the reported energy, and the
replicas' state is what the oracle gives after the same number of mega-iterations)."""
import time

import numpy as np
import pytest

import instances
from helpers import compare_solver_to_oracle, oracle_after

pytestmark = pytest.mark.gpu


def perm_energy(inst, perm):
    return int((inst.D.astype(np.int64) * inst.F[np.ix_(perm, perm)]).sum())


# launch_mode 1: the host tests the time between graph launches; 2: the persistent launch stops
# at the next mega-iteration boundary once the host sets its kill word
@pytest.mark.parametrize("mode", [1, 2])
def test_timeout_ends_an_unlimited_solve(gpu, mode):
    inst = instances.uniform(40, 401)
    p = gpu.default_params(replicas=8, groups=2, sweeps_per_exchange=4, beta_max=0.05, beta_ratio=1.3,
                           seed=3, timeout_s=0.2, max_megaiters=2 ** 40, megaiters_per_launch=16,
                           launch_mode=mode)
    t0 = time.perf_counter()
    r = gpu.solve(inst.F, inst.D, p)
    wall = time.perf_counter() - t0
    assert r["stopped_by"] == 2
    assert 0 < r["megaiters_done"] < p.max_megaiters
    assert wall < 0.2 + 10.0
    assert r["updates"] == r["megaiters_done"] * 4 * 40 * 16
    assert perm_energy(inst, r["best_perm"]) == r["best_energy"]


@pytest.mark.parametrize("mode", [1, 2])
def test_timeout_state_matches_the_oracle(gpu, oracle, mode):
    """The mega-iterations a timed-out run completed are ordinary ones: the full replica and
    group state equals the oracle's after that many mega-iterations, and a later run call
    continues from there."""
    inst = instances.uniform(20, 402)
    kw = dict(replicas=4, groups=2, sweeps_per_exchange=2, beta_max=0.05, beta_ratio=1.4, seed=5)
    p = gpu.default_params(timeout_s=0.05, max_megaiters=2 ** 40, megaiters_per_launch=4, launch_mode=mode, **kw)
    with gpu.Solver(inst.F, inst.D, p) as s:
        s.run(2 ** 40)
        first = s.result()["megaiters_done"]
        assert 0 < first
        s.run(2 ** 40)                       # a second call runs on after the first one's stop
        done = s.result()["megaiters_done"]
        assert done > first and s.result()["stopped_by"] == 0
        st = oracle_after(oracle, inst.F, inst.D, T=2, R=4, spe=2, beta_max=0.05, beta_ratio=1.4,
                          seed=5, cap=10, megaiters=done)
        bad = compare_solver_to_oracle(s, st, 10)
    assert not bad, bad[:5]


def test_timeout_after_the_last_megaiteration_is_not_a_timeout_stop(gpu):
    inst = instances.uniform(16, 403)
    p = gpu.default_params(replicas=4, groups=1, beta_max=0.05, seed=2, timeout_s=600.0, max_megaiters=5)
    r = gpu.solve(inst.F, inst.D, p)
    assert r["stopped_by"] == 0 and r["megaiters_done"] == 5
