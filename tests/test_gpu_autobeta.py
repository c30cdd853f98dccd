"""Automatic beta selection (the reference's default mode) on the GPU against the oracle.

The 160 trials run as one batched launch; their final energies, the 32 averages and the
selected beta0 / deltaBeta must equal the oracle restatement exactly.
"""
import numpy as np
import pytest

import instances
from helpers import oracle_auto_beta

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,T,R,spe", [(12, 2, 4, 2), (20, 1, 6, 1)])
def test_auto_beta_matches_oracle(gpu, oracle, n, T, R, spe):
    inst = instances.uniform(n, 500 + n)
    p = gpu.default_params(replicas=R, groups=T, sweeps_per_exchange=spe, seed=42)
    got = gpu.auto_beta(inst.F, inst.D, p)
    b0, db, sums, best = oracle_auto_beta(oracle, inst.F, inst.D, T=T, R=R, spe=spe, seed=42, cap=10)
    assert np.array_equal(got["avg_energy"], np.array(sums))
    assert got["beta0"] == b0
    assert got["delta_beta"] == db
    assert got["best_energy"] == best


def test_solve_in_automatic_mode_uses_the_selected_ladder(gpu):
    inst = instances.uniform(16, 601)
    p = gpu.default_params(replicas=4, groups=2, sweeps_per_exchange=2, seed=7, max_megaiters=20)
    sel = gpu.auto_beta(inst.F, inst.D, p)
    p.auto_beta = 1
    r = gpu.solve(inst.F, inst.D, p)
    assert r["beta_max_used"] == sel["beta0"] and r["beta_ratio_used"] == sel["delta_beta"]
    q = gpu.default_params(replicas=4, groups=2, sweeps_per_exchange=2, seed=7, max_megaiters=20,
                           beta_internal=1, beta_max=sel["beta0"], beta_ratio=sel["delta_beta"])
    fixed = gpu.solve(inst.F, inst.D, q)
    assert r["best_energy"] == min(fixed["best_energy"], sel["best_energy"])
    assert r["accepts"] == fixed["accepts"]
