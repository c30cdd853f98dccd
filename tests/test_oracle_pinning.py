"""The oracle restatement against the reference's own CPU_PIM.cpp (CPU only).

oracle/build_ref.sh compiles the reference source, unmodified except for its capacity
constants, with an engine shim that feeds it the solver's Philox words.  The restatement must
then reproduce the reference's complete state bit for bit: permutations, force matrices,
energies, bests, betas, rank slots and timeSinceSwap.  Where the reference could not be
built, the committed golden fixtures (tests/golden) pin the oracle instead.
"""
import numpy as np
import pytest

import instances
from oracle import RefHarness, ref_available

pytestmark = pytest.mark.skipif(not ref_available("big"), reason="reference harness not built")

# (variant, n, T, R, numitera, beta0 (internal), deltaBeta, megaiters, seed, generator)
CASES = [
    ("stock", 12, 2, 4, 1, 14.4, 1.58, 60, 1, "uniform"),
    ("stock", 32, 1, 10, 1, 14.4269504089, 1.5849, 40, 7, "uniform"),   # the n=32 plain case
    ("stock", 20, 3, 6, 4, 0.5, 1.3, 20, 9, "uniform"),
    ("stock", 16, 1, 5, 2, 1e-6, 1.1, 20, 3, "uniform"),                   # hot: cutoff below INT_MIN
    ("stock", 10, 2, 10, 1, 40.0, 1.2, 160, 5, "uniform"),                 # cold: forced extreme swaps
    ("stock", 14, 1, 4, 1, 3.0, 1.4, 140, 11, "uniform"),                  # junk rank slot (R < 10)
    ("stock", 18, 2, 3, 3, 0.02, 1.5, 15, 13, "asym"),                     # asymmetric, signed, diagonal
    ("big", 40, 2, 8, 2, 0.05, 1.3, 6, 17, "uniform"),
    ("big", 256, 1, 2, 1, 0.002, 1.5, 1, 19, "grid"),                      # n = 256
    ("big", 100, 1, 3, 1, 0.0005, 2.0, 2, 23, "heavy_small"),
    ("stock", 1, 1, 2, 1, 1.0, 1.2, 5, 29, "uniform"),                    # n = 1: only the self move
    ("stock", 2, 2, 3, 2, 0.3, 1.3, 12, 31, "uniform"),                   # n = 2
    ("big", 64, 1, 4, 2, 0.05, 1.25, 4, 37, "binary"),                    # 0/1 flows (binary-flow kernel's domain)
    # the heavy-tailed workload unscaled (lognormal flows, 70 % zeros, Euclidean distances):
    # a full 4-sweep epoch at n = 180 and n = 256, the reference's own delta function on it
    ("big", 180, 1, 2, 4, 1.2e-4, 1.08, 2, 41, "heavy"),
    ("big", 256, 1, 2, 4, 1.2e-4, 1.5, 2, 43, "heavy"),
]


def int32_exact(inst):
    """True when every force entry, delta and energy the reference computes in int32
    (CPU_PIM.cpp:54, :62, :164-192, :225) fits.  |I[i][a]| <= B[i][a], the rearrangement
    bound of the sorted rows of D and F; a delta is at most 4 max|I| + 16 max|D| max|F|; and
    since sum_i I[i][phi(i)] = -2E, |E| <= 1/2 sum_i max_a B[i][a]."""
    D = np.abs(inst.D.astype(np.float64))
    F = np.abs(inst.F.astype(np.float64))
    srt = lambda M: -np.sort(-M, axis=1)
    B = srt(D) @ srt(F).T + srt(D.T) @ srt(F.T).T
    lim = 2 ** 31 - 1
    return 4 * B.max() + 16 * D.max() * F.max() < lim and 0.5 * B.max(axis=1).sum() < lim


def make(gen, n, seed):
    if gen == "uniform":
        return instances.uniform(n, seed)
    if gen == "grid":
        return instances.grid256(seed)
    if gen == "binary":
        rng = np.random.default_rng(seed)
        up = np.triu((rng.random((n, n)) < 0.36).astype(np.int64), 1)
        D = instances.uniform(n, seed + 1).D
        return instances.Instance(n, up + up.T, D)
    if gen == "heavy":
        return instances.heavy(n, seed)
    if gen == "heavy_small":
        # heavy-tailed shape with flows scaled down so every int32 intermediate of the
        # reference stays exact
        inst = instances.heavy(n, seed)
        return instances.Instance(n, np.minimum(inst.F, 60), inst.D // 4)
    rng = np.random.default_rng(seed)
    return instances.Instance(n, rng.integers(-5, 40, (n, n)), rng.integers(-3, 60, (n, n)))


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}-n{c[1]}-T{c[2]}-R{c[3]}-i{c[4]}-{c[9]}" for c in CASES])
def test_restatement_matches_reference(oracle, case):
    variant, n, T, R, it, b0, db, M, seed, gen = case
    ref = RefHarness(variant)
    inst = make(gen, n, seed)
    assert int32_exact(inst), "the reference's int32 arithmetic would not be exact on this instance"
    ref.load(inst.F, inst.D)
    ref.setup(T, R, it, b0, db, seed)
    st = oracle.setup(inst.D, inst.F, T, R, it, b0, db, seed, cap=ref.maxr)
    for t in range(T):
        for l in range(R):
            r = ref.replica(t, l)
            assert np.array_equal(r["phi"], st.phi[t, l])
            assert np.array_equal(r["I"], st.I[t, l])
            assert r["E"] == st.E[t, l]
            assert r["beta"] == st.beta[t, l]
    ref.run(M)
    saw_forced = False
    for _ in range(M):
        oracle.run(st, inst.D, inst.F, 1)
        saw_forced |= bool((st.time_since_swap > 100).any())
    for t in range(T):
        g = ref.group(t)
        assert np.array_equal(g["order"], st.order[t])
        assert g["time_since_swap"] == st.time_since_swap[t]
        assert g["thread_best"] == st.thread_best[t]
        for l in range(R):
            r = ref.replica(t, l)
            assert np.array_equal(r["phi"], st.phi[t, l]), (t, l)
            assert np.array_equal(r["phiinv"], st.phiinv[t, l]), (t, l)
            assert np.array_equal(r["I"], st.I[t, l]), (t, l)
            assert (r["E"], r["bestE"], r["beta"]) == (st.E[t, l], st.bestE[t, l], st.beta[t, l])
    assert ref.single_best() == st.single_best
    if M > 120 and b0 >= 3.0:
        assert saw_forced, "expected the forced extreme swap path to be exercised"


def test_reference_file_reader_matches(tmp_path):
    """The reference's readProblem() reads what instances.write_instance writes."""
    ref = RefHarness("big")
    inst = instances.uniform(37, 5)
    path = str(tmp_path / "u37.dat")
    instances.write_instance(path, inst)
    assert ref.read_file(path) == 0
    F, D = ref.instance()
    assert np.array_equal(F, inst.F) and np.array_equal(D, inst.D)
    back = instances.read_instance(path)
    assert np.array_equal(back.F, inst.F) and np.array_equal(back.D, inst.D)


# (n = 256, 92 active facilities are hard-wired in the reference's tai256c program)
TAI_CASES = [
    (2, 3, 1, 0.002, 1.5, 2, 29),
    (1, 4, 2, 0.02, 1.3, 2, 31),          # colder: the lumped candidate dominates inactive picks
]


@pytest.mark.skipif(not ref_available("tai"), reason="reference tai256c harness not built")
@pytest.mark.parametrize("case", TAI_CASES, ids=[f"T{c[0]}-R{c[1]}-i{c[2]}-b{c[3]}" for c in TAI_CASES])
def test_clique_restatement_matches_reference_tai256c(oracle, case):
    """orc_update_clique against CPU_PIM_tai256c.cpp (doMegaIteraTai) on a 92-clique instance."""
    T, R, it, b0, db, M, seed = case
    ref = RefHarness("tai")
    inst = instances.clique_flow(seed)
    ref.load(inst.F, inst.D)
    ref.setup(T, R, it, b0, db, seed)
    st = oracle.setup(inst.D, inst.F, T, R, it, b0, db, seed, cap=ref.maxr, active=92)
    before = st.phi.copy()
    ref.run(M)
    oracle.run(st, inst.D, inst.F, M)
    moved_inactive = 0
    for t in range(T):
        g = ref.group(t)
        assert np.array_equal(g["order"], st.order[t])
        assert g["thread_best"] == st.thread_best[t]
        for l in range(R):
            r = ref.replica(t, l)
            assert np.array_equal(r["phi"], st.phi[t, l]), (t, l)
            assert np.array_equal(r["I"], st.I[t, l]), (t, l)
            assert (r["E"], r["bestE"], r["beta"]) == (st.E[t, l], st.bestE[t, l], st.beta[t, l])
            moved_inactive += int(((before[t, l] >= 92) & (st.phi[t, l] >= 92) & (before[t, l] != st.phi[t, l])).sum())
    assert moved_inactive > 0, "expected lumped inactive-to-inactive moves"
