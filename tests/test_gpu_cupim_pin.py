"""The one-shot rule's oracle pinned against the reference's own one-shot kernels.

The one-shot rule is GPU-CUPIM's step (perl-gpu/src/lib/qap/qap.cu:1462-1600: os_pwc_d
proposals, the os_resolve_* ballot race, os_update_force_mats_d, os_apply_swaps_ii_d and
os_score_from_force_mat_d).  oracle/build_cupim.sh compiles that source as it lies into
oracle/_ref/libref_cupim.so with one substitution: its cuRANDDx generator (mathdx, not vendored
with the reference) is replaced by one that copies the uniforms the oracle draws
(oracle/cupim_shim/random.cuh).  This test runs the reference's kernels and the oracle's
restatement (orc_oneshot_step) side by side from the same permutations, betas and uniforms and
requires, after the reference's set-up and after every step, the same permutation, force matrix
and energy of every replica, and the same partner for every proposal the reference applied or
kept as a self move.

The oracle's binary32 weights come from the project's own 2^x (under 1 ulp), the reference's
from CUDA's exp2f; a decision can only differ when u * total falls within a few ulp of a
prefix boundary, which these fixed seeds do not hit (tolerance: zero mismatches on the cases
below; the rate over long streams is measured by bench.py --suite divergence --update-rule
one-shot).  The solver with oneshot_weights = 1 equals the oracle bit for bit
(tests/test_gpu_oneshot.py); with the default oneshot_weights = 0 it computes the weights with
CUDA's exp2f exactly as the reference writes them, and the second test below requires its
trajectories to equal the reference kernels' (tolerance: zero mismatches).
"""
import os

import numpy as np
import pytest

import instances
from test_gpu_parity import asym, binary

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref_cupim.so")

# name: (instance factory, replicas, coldest beta (as used in 2^(beta dE)), ladder ratio, steps)
CASES = {
    "uniform_n32": (lambda: instances.uniform(32, 11), 8, 2e-3, 2.0, 12),
    "asym_signed_n18": (lambda: asym(18, 13), 4, 0.02, 2.0, 12),
    "asym_odd_n37": (lambda: asym(37, 29), 3, 0.01, 3.0, 10),
    "binary_n90": (lambda: binary(90, 32), 4, 0.02, 2.0, 8),
    "uniform_n200": (lambda: instances.uniform(200, 19), 2, 2e-3, 4.0, 6),
    "uniform_n250_even": (lambda: instances.uniform(250, 31), 2, 2e-3, 4.0, 5),
    "grid_n256": (lambda: instances.grid256(17), 4, 0.004, 2.0, 6),
    "hot_collisions_n16": (lambda: instances.uniform(16, 22), 4, 1e-6, 2.0, 12),
    "n5_tiny": (lambda: instances.uniform(5, 25), 3, 0.05, 2.0, 12),
    "n1_trivial": (lambda: instances.uniform(1, 24), 2, 1.0, 2.0, 3),
}


@pytest.fixture(scope="module")
def cupim():
    if not os.path.exists(LIB):
        pytest.skip("oracle/_ref/libref_cupim.so not built (the reference source was absent at build time)")
    from oracle import CupimRef
    return CupimRef(LIB)


@pytest.mark.parametrize("name", list(CASES))
def test_oneshot_oracle_matches_reference_kernels(cupim, oracle, tmp_path, name):
    make, R, bcold, ratio, steps = CASES[name]
    inst = make()
    n = inst.n
    D = np.ascontiguousarray(inst.D, np.int32)
    F = np.ascontiguousarray(inst.F, np.int32)
    path = str(tmp_path / "inst.dat")
    instances.write_instance(path, inst)
    seed = 0x5EED0000 + n
    rng = np.random.default_rng(n)
    phi0 = np.stack([rng.permutation(n) for _ in range(R)]).astype(np.int32)
    betas = np.array([bcold / ratio ** r for r in range(R)], np.float32)

    cupim.open(path, R)
    try:
        cupim.set(phi0, betas)
        # the oracle's replicas from the same permutations
        I, phi, inv, E, bestE = [], [], [], [], []
        for r in range(R):
            Ir, Er = oracle.force_init(D, F, phi0[r])
            I.append(Ir)
            p = phi0[r].copy()
            q = np.zeros(n, np.int32)
            q[p] = np.arange(n, dtype=np.int32)
            phi.append(p)
            inv.append(q)
            E.append(np.array([Er], np.int64))
            bestE.append(np.array([Er], np.int64))
        _, cforce, cscore, _ = cupim.get()
        for r in range(R):
            assert np.array_equal(cforce[r], I[r]), f"replica {r}: set-up force matrix"
            assert int(cscore[r]) == int(E[r][0]), f"replica {r}: set-up energy"
        compared = applied = 0
        for s in range(steps):
            # replica r of the pool is replica r of group 0 of the oracle's stream
            cupim.step(oracle.oneshot_uniforms(seed, R, R, s, n))
            cphi, cforce, cscore, ctg = cupim.get()
            for r in range(R):
                nsw, tg = oracle.oneshot_step(D, F, I[r], phi[r], inv[r], E[r], bestE[r], float(betas[r]),
                                              seed, 0, r, s)
                where = f"step {s} replica {r}"
                kept = ctg[r] < n                        # applied swaps and self proposals
                assert np.array_equal(ctg[r][kept], tg[kept]), f"{where}: proposals"
                assert np.array_equal(cphi[r], phi[r]), f"{where}: permutation"
                assert np.array_equal(cforce[r], I[r]), f"{where}: force matrix"
                assert int(cscore[r]) == int(E[r][0]), f"{where}: energy"
                compared += n
                applied += nsw
        if n > 1 and name != "n5_tiny":
            assert applied > 0
        print(f"{name}: {compared} proposals, {applied} swaps applied, all equal")
    finally:
        cupim.close()


# The solver itself against the reference's kernels, without the oracle: groups of one replica
# (rank_slots 1, so the exchange never moves a beta) run the one-shot rule on the GPU, and the
# reference's pool, one replica per group, takes the same steps from the solver's initial
# permutations with the solver's thresholds; the permutations and energies are compared after
# every mega-iteration chunk.
SOLVER_CASES = {
    "grid_n256_cold": (lambda: instances.grid256(1000), 16, 2.0 ** -5, 4, 3),
    "grid_n256_hot": (lambda: instances.grid256(1001), 16, 2.0 ** -10, 4, 3),
    "uniform_n32": (lambda: instances.uniform(32, 77), 32, 2.0 ** -9, 4, 5),
    "asym_n70": (lambda: asym(70, 78), 8, 0.004, 2, 4),
}


@pytest.mark.parametrize("name", list(SOLVER_CASES))
def test_oneshot_solver_matches_reference_kernels(cupim, oracle, gpu, tmp_path, name):
    make, G, beta, spe, chunks = SOLVER_CASES[name]
    inst = make()
    n = inst.n
    path = str(tmp_path / "inst.dat")
    instances.write_instance(path, inst)
    seed = 4242
    p = gpu.default_params(replicas=1, groups=G, rank_slots=1, sweeps_per_exchange=spe, beta_max=beta,
                           beta_ratio=1.5, beta_internal=1, seed=seed, max_megaiters=2 ** 31 - 1,
                           megaiters_per_launch=2, update_rule=gpu.RULE_ONE_SHOT, goal=-(1 << 62))
    betas = np.full(G, np.float32(beta), np.float32)
    cupim.open(path, G)
    try:
        with gpu.Solver(inst.F, inst.D, p) as s:
            phi0 = np.stack([s.replica(g, 0, force=False)["phi"] for g in range(G)]).astype(np.int32)
            cupim.set(phi0, betas)
            step = 0
            for c in range(chunks):
                s.run(2)
                for _ in range(2 * spe):
                    cupim.step(oracle.oneshot_uniforms(seed, G, 1, step, n))
                    step += 1
                cphi, _, cscore, _ = cupim.get(force=False)
                for g in range(G):
                    r = s.replica(g, 0, force=False)
                    assert np.array_equal(r["phi"], cphi[g]), f"chunk {c} group {g}: permutation"
                    assert r["E"] == int(cscore[g]), f"chunk {c} group {g}: energy"
            print(f"{name}: {G * step * n} proposals, all equal")
    finally:
        cupim.close()
