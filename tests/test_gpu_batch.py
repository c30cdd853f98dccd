"""GPU parity of the batched solve: one persistent launch over many instances of uneven n.

Every instance of a batch must end exactly where pimqap_solve leaves it when it runs alone
(same best energy, permutation, accepted-swap count, mega-iterations and goal stop), and a
subset is checked against the oracle directly.
"""
import numpy as np
import pytest

import instances
from helpers import oracle_after

pytestmark = pytest.mark.gpu


def asym(n, seed):
    rng = np.random.default_rng(seed)
    return instances.Instance(n, rng.integers(-5, 40, (n, n)), rng.integers(-3, 60, (n, n)))


def same(a, b):
    keys = ("best_energy", "megaiters_done", "updates", "sweeps", "proposals", "accepts", "target_megaiter",
            "stopped_by")
    return all(a[k] == b[k] for k in keys) and np.array_equal(a["best_perm"], b["best_perm"])


def mixed_batch(gpu):
    insts, params = [], []
    rng = np.random.default_rng(5)
    for k in range(24):
        n = int(rng.integers(5, 150))
        inst = instances.uniform(n, 900 + k) if k % 5 else asym(n, 900 + k)
        insts.append(inst)
        params.append(gpu.default_params(replicas=int(rng.integers(2, 9)), groups=1 + k % 3,
                                         sweeps_per_exchange=1 + k % 4, beta_max=0.02 + 0.01 * (k % 3),
                                         beta_ratio=1.3, seed=1000 + k,
                                         max_megaiters=int(rng.integers(1, 12))))
    # an int64 instance, a cluster-sized one, and one that stops on its goal
    insts.append(instances.Instance(30, rng.integers(0, 2_000_000, (30, 30)), rng.integers(0, 5000, (30, 30))))
    params.append(gpu.default_params(replicas=3, groups=2, sweeps_per_exchange=2, beta_max=1e-9,
                                     beta_ratio=1.5, seed=77, max_megaiters=5))
    insts.append(instances.grid256(901))
    params.append(gpu.default_params(replicas=2, groups=1, sweeps_per_exchange=1, beta_max=0.0015,
                                     beta_ratio=1.5, seed=78, max_megaiters=2))
    # int64 force matrices that need a 2-CTA and a 4-CTA cluster
    for n, seed in ((180, 903), (250, 904)):
        insts.append(instances.Instance(n, rng.integers(0, 2_000_000, (n, n)), rng.integers(0, 5000, (n, n))))
        params.append(gpu.default_params(replicas=2, groups=1, sweeps_per_exchange=1, beta_max=1e-9,
                                         beta_ratio=1.5, seed=seed, max_megaiters=2))
    goal_inst = instances.uniform(24, 902)
    probe = gpu.solve(goal_inst.F, goal_inst.D, gpu.default_params(
        replicas=6, groups=2, sweeps_per_exchange=1, beta_max=0.05, beta_ratio=1.3, seed=79,
        max_megaiters=40))
    insts.append(goal_inst)
    params.append(gpu.default_params(replicas=6, groups=2, sweeps_per_exchange=1, beta_max=0.05,
                                     beta_ratio=1.3, seed=79, max_megaiters=60,
                                     goal=probe["best_energy"] + 600))
    return insts, params


def test_batch_equals_individual_solves(gpu):
    insts, params = mixed_batch(gpu)
    got = gpu.batch_solve([(i.F, i.D) for i in insts], params)
    assert got[-1]["stopped_by"] == 1
    for k, (inst, p) in enumerate(zip(insts, params)):
        alone = gpu.solve(inst.F, inst.D, p)
        assert same(got[k], alone), (k, inst.n, got[k], alone)


def test_batch_matches_oracle(gpu, oracle):
    cases = [(instances.uniform(17, 950), 2, 3, 2, 0.04, 1.3, 9),
             (asym(33, 951), 1, 4, 1, 0.01, 1.4, 6),
             (instances.uniform(64, 952), 3, 2, 3, 0.005, 1.6, 4)]
    params = [gpu.default_params(replicas=R, groups=T, sweeps_per_exchange=spe, beta_max=b,
                                 beta_ratio=m, seed=60 + k, max_megaiters=M)
              for k, (_, T, R, spe, b, m, M) in enumerate(cases)]
    got = gpu.batch_solve([(c[0].F, c[0].D) for c in cases], params)
    for k, (inst, T, R, spe, b, m, M) in enumerate(cases):
        st = oracle_after(oracle, inst.F, inst.D, T=T, R=R, spe=spe, beta_max=b, beta_ratio=m,
                          seed=60 + k, cap=10, megaiters=M)
        assert got[k]["accepts"] == st.accepts
        assert got[k]["best_energy"] == min(int(st.bestE.min()), st.single_best)
        assert got[k]["megaiters_done"] == M


def test_same_result_alone_and_in_a_mix(gpu):
    """A request's result does not depend on what else is in the launch."""
    target = instances.uniform(45, 960)
    p = gpu.default_params(replicas=8, groups=2, sweeps_per_exchange=2, beta_max=0.02,
                           beta_ratio=1.3, seed=5, max_megaiters=10)
    alone = gpu.batch_solve([(target.F, target.D)], [p])[0]
    others = [instances.uniform(int(n), 961 + j) for j, n in enumerate((20, 150, 90, 33, 120))]
    mix = [(o.F, o.D) for o in others[:3]] + [(target.F, target.D)] + [(o.F, o.D) for o in others[3:]]
    ps = [gpu.default_params(replicas=4, groups=1, sweeps_per_exchange=1, beta_max=0.03,
                             beta_ratio=1.3, seed=j, max_megaiters=7) for j in range(6)]
    ps[3] = p
    got = gpu.batch_solve(mix, ps)[3]
    assert same(got, alone)


def test_heavy_batch_matches_solo_and_oracle(gpu, oracle):
    """Eight instances of the heavy-tailed 128-instance batch (n ~ U[100, 256], lognormal flows
    with 70 % zeros, Euclidean distances) in one launch on the heavy ladder: each equals its
    solo solve, and its complete replica state equals the oracle's."""
    from helpers import compare_solver_to_oracle
    batch = instances.heavy_batch(8)
    b0 = 2.0 ** -13 / 1.44269504089
    params = [gpu.default_params(replicas=4, groups=1, sweeps_per_exchange=4, beta_max=b0, beta_ratio=1.5,
                                 seed=500 + k, max_megaiters=2) for k in range(len(batch))]
    got = gpu.batch_solve([(b.F, b.D) for b in batch], params)
    for k, (inst, p) in enumerate(zip(batch, params)):
        alone = gpu.solve(inst.F, inst.D, p)
        assert same(got[k], alone), (k, inst.n)
        st = oracle_after(oracle, inst.F, inst.D, T=1, R=4, spe=4, beta_max=b0, beta_ratio=1.5,
                          seed=500 + k, cap=10, megaiters=2)
        assert got[k]["accepts"] == st.accepts
        assert got[k]["best_energy"] == min(int(st.bestE.min()), st.single_best)
        with gpu.Solver(inst.F, inst.D, p) as s:   # the full state, through the solver handle
            s.run(2)
            bad = compare_solver_to_oracle(s, st, 10)
        assert not bad, (k, bad[:5])


def test_autotuner_choice_is_no_slower_and_changes_no_result(gpu, monkeypatch):
    """The autotuner times every candidate worker shape of a class, the fixed rules' shape among
    them, and keeps the fastest; results are the same with its shapes and with the fixed rules'."""
    batch = instances.uniform_batch(48, n_lo=20, n_hi=150, seed=11)
    params = [gpu.default_params(replicas=8, groups=1, sweeps_per_exchange=2, beta_max=0.02, beta_ratio=1.3,
                                 seed=70 + k, max_megaiters=3) for k in range(len(batch))]
    pairs = [(b.F, b.D) for b in batch]
    report = gpu.batch_tune(pairs, params)
    assert report
    for c in report:
        assert c["members"] > 0 and c["threads"] >= 32 and c["workers"] >= 1 and c["grid"] >= 1
        if c["tried"] > 1:
            assert c["tuned_ms"] <= c["fixed_ms"], c
    tuned = gpu.batch_solve(pairs, params)
    monkeypatch.setenv("PIMQAP_AUTOTUNE", "0")
    rules = gpu.batch_solve(pairs, params)
    off = gpu.batch_tune(pairs, params)
    assert all(c["tried"] == 0 and (c["threads"], c["workers"]) == (c["fixed_threads"], c["fixed_workers"])
               for c in off)
    for k, (a, b) in enumerate(zip(tuned, rules)):
        assert same(a, b), k


def test_cached_shape_is_not_applied_where_it_does_not_fit(gpu):
    """The autotuner caches a class's shape by its largest n in buckets of 16; a batch whose
    largest n is in the same bucket but needs a larger worker slice must not inherit a worker
    count that overflows a CTA's shared memory (it keeps its own fixed-rule shape)."""
    def batch(ns, seed):
        insts = [instances.uniform(n, seed + k) for k, n in enumerate(ns)]
        ps = [gpu.default_params(replicas=8, groups=1, sweeps_per_exchange=1, beta_max=0.02, beta_ratio=1.3,
                                 seed=seed + k, max_megaiters=2) for k in range(len(ns))]
        return insts, ps
    small, ps = batch([150, 145, 153, 149] * 6, 700)
    gpu.batch_tune([(i.F, i.D) for i in small], ps)
    big, qs = batch([158, 157, 156, 155] * 6, 800)
    got = gpu.batch_solve([(i.F, i.D) for i in big], qs)
    for k, (inst, p) in enumerate(zip(big[:4], qs[:4])):
        assert same(got[k], gpu.solve(inst.F, inst.D, p)), k
