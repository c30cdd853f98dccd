"""GPU parity of the one-shot update rule (GPU-CUPIM's os_* step, qap.cu:1038-1458): the CUDA
solver through its C ABI against the oracle restatement (orc_oneshot_step).

Everything is bit-exact: permutations, force matrices, energies, bests, betas, rank slots,
accept counts.  The solver runs with oneshot_weights = 1, the library's own binary32 2^x,
which the oracle restates (checked bit for bit below); every other floating-point step is a
single IEEE operation in the same order, so the proposals agree exactly (tolerance: zero
mismatches).  The default weights (CUDA's exp2f, as the reference computes them) are compared
with the reference's own kernels in tests/test_gpu_cupim_pin.py.
"""
import numpy as np
import pytest

import instances
from helpers import compare_solver_to_oracle, oracle_after
from test_gpu_parity import asym, binary, heavy_small, wide

pytestmark = pytest.mark.gpu

# name: (instance factory, T, R, spe, beta_max (natural), beta_ratio, megaiters, extra params)
CASES = {
    "plain_n32_R16": (lambda: instances.uniform(32, 11), 1, 16, 1, 10.0, 1.5849, 25, {}),
    "groups_T3_R5_i4": (lambda: instances.uniform(20, 12), 3, 5, 4, 0.4, 1.3, 8, {}),
    "asym_signed_n18": (lambda: asym(18, 13), 2, 3, 3, 0.015, 1.5, 10, {}),
    "int64_forced_n24": (lambda: instances.uniform(24, 14), 1, 4, 2, 0.01, 1.4, 10, {"force_bits": 64}),
    "heavy_n60": (lambda: heavy_small(60, 15), 1, 3, 1, 0.0005, 2.0, 6, {}),
    "wide_int64_n32": (lambda: wide(32, 26), 2, 3, 2, 1e-9, 1.5, 6, {}),
    "grid_n256_cluster2": (lambda: instances.grid256(17), 1, 2, 1, 0.0015, 1.5, 3, {}),
    "grid_n256_int64_cluster4": (lambda: instances.grid256(18), 1, 1, 1, 0.0015, 1.5, 2, {"force_bits": 64}),
    "n200": (lambda: instances.uniform(200, 19), 1, 2, 1, 0.0005, 1.5, 2, {}),
    "cold_forced_swaps": (lambda: instances.uniform(12, 20), 2, 10, 1, 40.0, 1.2, 150, {}),
    "hot_collisions": (lambda: instances.uniform(16, 22), 1, 5, 2, 1e-6, 1.1, 10, {}),
    "threads64_n40": (lambda: instances.uniform(40, 23), 1, 4, 2, 0.02, 1.3, 6, {"threads_per_block": 64}),
    # n = 1 has energy 0, and this rule tracks the best after every step: a goal below 0 keeps
    # the run going (with the default goal 0 it stops after the first tracking)
    "n1_trivial": (lambda: instances.uniform(1, 24), 1, 2, 1, 1.0, 1.2, 3, {"goal": -1}),
    "n5_tiny": (lambda: instances.uniform(5, 25), 2, 3, 2, 0.05, 1.3, 6, {}),
    "asym_n70_cluster2": (lambda: asym(70, 28), 1, 3, 2, 0.002, 1.5, 3, {"cluster_size": 2}),
    "asym_n37_cluster4_t64": (lambda: asym(37, 29), 2, 2, 1, 0.003, 1.5, 4,
                              {"cluster_size": 4, "threads_per_block": 64}),
    "n250_cluster4_ragged": (lambda: instances.uniform(250, 31), 1, 2, 1, 0.0005, 1.5, 2, {"cluster_size": 4}),
    "binary_n90": (lambda: binary(90, 32), 2, 3, 2, 0.01, 1.4, 4, {}),
    "goal_print_events": (lambda: instances.uniform(30, 36), 1, 4, 2, 0.02, 1.3, 6,
                          {"goal_print": 10 ** 9, "event_capacity": 4096}),
}


def run_case(gpu, oracle, name, seed=7, more=None):
    make, T, R, spe, bmax, ratio, M, extra = CASES[name]
    extra = dict(extra, **(more or {}))
    inst = make()
    cap = max(R, 10)
    p = gpu.default_params(replicas=R, groups=T, sweeps_per_exchange=spe, beta_max=bmax,
                           beta_ratio=ratio, seed=seed, max_megaiters=M, megaiters_per_launch=7,
                           update_rule=gpu.RULE_ONE_SHOT, oneshot_weights=1, **extra)
    with gpu.Solver(inst.F, inst.D, p) as s:
        s.run(M)
        st = oracle_after(oracle, inst.F, inst.D, T=T, R=R, spe=spe, beta_max=bmax,
                          beta_ratio=ratio, seed=seed, cap=cap, megaiters=M, rule=1,
                          goal=extra.get("goal", 0))
        bad = compare_solver_to_oracle(s, st, cap)
        res = s.result()
        events = s.events() if extra.get("event_capacity") else []
    return inst, st, bad, res, events


@pytest.mark.parametrize("name", list(CASES))
def test_oneshot_trajectory_matches_oracle(gpu, oracle, name):
    inst, st, bad, res, events = run_case(gpu, oracle, name)
    assert not bad, bad[:10]
    assert res["megaiters_done"] == CASES[name][6]
    assert res["accepts"] == st.accepts
    assert res["best_energy"] == min(int(st.bestE.min()), st.single_best)
    if inst.n > 1 and name != "cold_forced_swaps":
        assert st.accepts > 0
    if name == "goal_print_events":
        assert any(e["kind"] == gpu.EVENT_GOAL_PRINT for e in events)


# the force update on the integer CUDA cores (1), by mma.sync (2) and by tcgen05 with the sums in
# tensor memory (3): symmetric and asymmetric (two factor columns per swap), clusters of 1, 2
# and 4 (rows per CTA 256 / 2, 250 / 4 ragged), N = 16 .. 256, steps of many swaps (hot ladders)
FORM_CASES = ["plain_n32_R16", "groups_T3_R5_i4", "asym_signed_n18", "grid_n256_cluster2",
              "n250_cluster4_ragged", "asym_n70_cluster2", "binary_n90", "n5_tiny", "hot_collisions",
              "n1_trivial", "n200", "cold_forced_swaps"]


@pytest.mark.parametrize("form", [1, 2, 3])
@pytest.mark.parametrize("name", FORM_CASES)
def test_force_update_forms_match_oracle(gpu, oracle, name, form):
    inst, st, bad, res, _ = run_case(gpu, oracle, name, more={"tensor_update": form})
    assert not bad, bad[:10]
    assert res["accepts"] == st.accepts
    assert res["best_energy"] == min(int(st.bestE.min()), st.single_best)


def test_tcgen05_form_rejected_where_inexact_or_unshaped(gpu):
    big = instances.uniform(30, 9)   # flows scaled past 2048: fp16 cannot hold every factor
    F = np.ascontiguousarray(big.F * 40)
    p = gpu.default_params(replicas=2, groups=1, beta_max=0.00001, max_megaiters=1,
                           update_rule=gpu.RULE_ONE_SHOT, tensor_update=3)
    with pytest.raises(gpu.PimqapError) as e:
        gpu.solve(F, big.D, p)
    assert "tensor_update" in str(e.value)
    p.tensor_update = 2
    with pytest.raises(gpu.PimqapError):
        gpu.solve(F, big.D, p)
    p.tensor_update = 0                # automatic: the integer CUDA cores
    assert gpu.solve(F, big.D, p)["megaiters_done"] == 1
    inst = instances.uniform(40, 23)
    p = gpu.default_params(replicas=2, groups=1, beta_max=0.02, max_megaiters=1,
                           update_rule=gpu.RULE_ONE_SHOT, tensor_update=3, threads_per_block=64)
    with pytest.raises(gpu.PimqapError) as e:
        gpu.solve(inst.F, inst.D, p)
    assert "tcgen05" in str(e.value)
    # automatic: the same instance and shape run (on mma.sync)
    p.tensor_update = 0
    assert gpu.solve(inst.F, inst.D, p)["megaiters_done"] == 1


def test_tcgen05_many_small_ctas_per_sm(gpu, oracle):
    """n = 24 (32 tensor-memory columns per CTA), 64 groups x 16 replicas: 1024 single-CTA
    replicas of 128 threads, several per SM, each holding tensor memory for its whole epoch."""
    inst = instances.uniform(24, 41)
    T, R, spe, M = 64, 16, 1, 3
    p = gpu.default_params(replicas=R, groups=T, sweeps_per_exchange=spe, beta_max=10.0,
                           beta_ratio=1.5849, seed=3, max_megaiters=M, update_rule=gpu.RULE_ONE_SHOT,
                           tensor_update=3, oneshot_weights=1)
    with gpu.Solver(inst.F, inst.D, p) as s:
        s.run(M)
        st = oracle_after(oracle, inst.F, inst.D, T=T, R=R, spe=spe, beta_max=10.0, beta_ratio=1.5849,
                          seed=3, cap=max(R, 10), megaiters=M, rule=1)
        bad = compare_solver_to_oracle(s, st, max(R, 10))
    assert not bad, bad[:10]


def test_oneshot_shapes(gpu, oracle):
    _, _, _, r, _ = run_case(gpu, oracle, "grid_n256_cluster2")
    assert (r["force_bits"], r["cluster_size"]) == (32, 2)
    _, _, _, r, _ = run_case(gpu, oracle, "grid_n256_int64_cluster4")
    assert (r["force_bits"], r["cluster_size"]) == (64, 4)


def test_weight_exp2_bits_match_oracle(gpu, oracle):
    """The device's binary32 exp2 returns the oracle's bits on every input tried."""
    rng = np.random.default_rng(5)
    x = np.concatenate([
        -rng.random(200000, dtype=np.float32) * 152.0,
        -rng.random(100000, dtype=np.float32) * 2.0,
        -np.arange(0, 152, 0.5, dtype=np.float32),
        np.float32([0.0, -0.0, -1e-30, -126.0, -126.5, -149.0, -149.5, -150.0, -1e30]),
    ]).astype(np.float32)
    y = gpu.probe_weight_exp2(x)
    ref = np.array([oracle.exp2f_neg(float(v)) for v in x], np.float32)
    mism = np.nonzero(y.view(np.uint32) != ref.view(np.uint32))[0]
    assert mism.size == 0, [(float(x[k]), float(y[k]), float(ref[k])) for k in mism[:10]]


def test_oneshot_rejected_where_unsupported(gpu):
    inst = instances.uniform(20, 3)
    p = gpu.default_params(replicas=3, groups=1, beta_max=0.05, max_megaiters=2,
                           update_rule=gpu.RULE_ONE_SHOT)
    with pytest.raises(gpu.PimqapError):
        gpu.batch_solve([(inst.F, inst.D)], [p])
    with pytest.raises(gpu.PimqapError):
        gpu.solve_static(inst.F, inst.D, p)
    p.auto_beta = 1
    with pytest.raises(gpu.PimqapError):
        gpu.solve(inst.F, inst.D, p)
    p.auto_beta = 0
    p.update_rule = 2
    with pytest.raises(gpu.PimqapError):
        gpu.solve(inst.F, inst.D, p)
