"""The one-shot parallel update of GPU-CUPIM (qap.cu:1038-1458) as the oracle restates it
(CPU only).

That reference code needs cuRANDDx and a GPU, so no reference output pins this restatement.
These tests pin it instead by (1) a second, independent restatement of the proposal's
lane-order scan in numpy binary32 arithmetic, (2) the exact identities every step must keep
(force matrix and energy equal to a fresh recomputation, disjoint swaps, the ballot rule),
and (3) the accuracy of the binary32 exp2 against the exact function.
"""
import numpy as np
import pytest

import instances

f32 = np.float32


def test_exp2f_neg_accuracy(oracle):
    rng = np.random.default_rng(3)
    xs = np.concatenate([-rng.random(20000) * 150, -rng.random(20000) * 4,
                         [0.0, -0.5, -1.0, -1.5, -125.5, -126.0, -126.49, -127.3, -149.9]]).astype(np.float32)
    for x in xs:
        y = oracle.exp2f_neg(float(x))
        t = 2.0 ** float(x)
        if t >= 2.0 ** -126:
            assert abs(y - t) <= 1.0 * float(np.spacing(f32(t))), (x, y, t)
        else:   # subnormal results: one rounding to the subnormal grid (spacing 2^-149)
            assert abs(y - t) <= 2.0 ** -149, (x, y, t)
    assert oracle.exp2f_neg(0.0) == 1.0
    assert oracle.exp2f_neg(-150.0) == 0.0 and oracle.exp2f_neg(-1e30) == 0.0
    assert oracle.exp2f_neg(-1.0) == 0.5 and oracle.exp2f_neg(-10.0) == 2.0 ** -10
    ys = [oracle.exp2f_neg(float(x)) for x in np.linspace(-30, 0, 5001).astype(np.float32)]
    assert all(b >= a for a, b in zip(ys, ys[1:]))          # monotone on an increasing grid


def test_oneshot_uniform(oracle):
    for w in (0, 1, 511, 512, 0xFFFFFFFF, 0x80000000, 123456789):
        u = oracle.oneshot_uniform(w)
        assert 0.0 < u < 1.0
        assert u == (((w >> 9) << 1) | 1) * 2.0 ** -24


def py_pick(oracle, d, beta_f, u):
    """The proposal of qap.cu:1040-1146 in numpy binary32, lane by lane."""
    n = len(d)
    mx = max(d)
    K = (n + 31) // 32
    s = np.zeros((32, K), np.float32)
    tot = np.zeros(32, np.float32)
    for t in range(32):
        run = f32(0)
        for k in range(K):
            j = t + 32 * k
            w = f32(oracle.exp2f_neg(float(f32(beta_f) * f32(d[j] - mx)))) if j < n else f32(0)
            run = w if k == 0 else f32(w + run)
            s[t, k] = run
        tot[t] = run
    x = tot.copy()
    dd = 1
    while dd < 32:
        y = x.copy()
        for t in range(dd, 32):
            y[t] = f32(x[t] + x[t - dd])
        x = y
        dd <<= 1
    off = (x - tot).astype(np.float32)
    total = f32(off[31] + tot[31])
    thresh = f32(f32(u) * total)
    for t in range(32):
        win = -1
        for k in range(K):
            j = t + 32 * k
            if j >= n:
                break
            cur = f32(off[t] + s[t, k])
            prev = off[t] if k == 0 else f32(off[t] + s[t, k - 1])
            if cur >= thresh and prev < thresh:
                win = j
        if win >= 0:
            return win, int(d[win])
    return n - 1, int(d[n - 1])


@pytest.mark.parametrize("n", [1, 5, 31, 32, 33, 70, 256])
def test_pick_matches_independent_restatement(oracle, n):
    rng = np.random.default_rng(n)
    for trial in range(40 if n < 200 else 8):
        d = rng.integers(-400, 60, n).astype(np.int64)
        d[rng.integers(0, n)] = 0                      # the self candidate
        beta_f = float(f32(10.0 ** rng.uniform(-4, 0)))
        u = oracle.oneshot_uniform(int(rng.integers(0, 2 ** 32)))
        assert oracle.oneshot_pick(d, beta_f, u) == py_pick(oracle, d, beta_f, u), (n, trial)


def test_pick_edges(oracle):
    # very cold: the first of the largest deltas in lane order takes every threshold
    d = np.array([0, -5, 7, 3, -2, 7], np.int64)
    assert oracle.oneshot_pick(d, 50.0, 0.5) == (2, 7)
    assert oracle.oneshot_pick(d, 50.0, 2.0 ** -24) == (2, 7)
    # equal weights over 40 partners: lanes 0-7 hold two (j and j + 32), so the prefix runs in
    # lane order and u = 0.999 lands in lane 31 (j = 31), not on j = 39 as a scan in j order would
    assert oracle.oneshot_pick(np.zeros(40, np.int64), 1.0, 0.999) == (31, 0)
    assert oracle.oneshot_pick(np.zeros(40, np.int64), 1.0, 0.01) == (0, 0)


def direct_energy(D, F, phi):
    return int((D * F[np.ix_(phi, phi)]).sum())


@pytest.mark.parametrize("gen,n,beta", [("uniform", 12, 0.003), ("uniform", 40, 0.02), ("asym", 23, 0.01),
                                        ("grid", 256, 0.002)])
def test_step_identities(oracle, gen, n, beta):
    if gen == "uniform":
        inst = instances.uniform(n, 5)
    elif gen == "grid":
        inst = instances.grid256(5)
    else:
        rng = np.random.default_rng(9)
        inst = instances.Instance(n, rng.integers(-5, 40, (n, n)), rng.integers(-3, 60, (n, n)))
    D = np.ascontiguousarray(inst.D, np.int32)
    F = np.ascontiguousarray(inst.F, np.int32)
    rng = np.random.default_rng(n)
    phi = rng.permutation(n).astype(np.int32)
    inv = np.argsort(phi).astype(np.int32)
    I, E0 = oracle.force_init(D, F, phi)
    E = np.array([E0], np.int64)
    bestE = np.array([2147483647], np.int64)
    total = 0
    for step in range(6 if n < 200 else 2):
        before = phi.copy()
        I_before = I.copy()
        swaps, tg = oracle.oneshot_step(D, F, I, phi, inv, E, bestE, beta, 77, 1, 2, step)
        total += swaps
        # the proposals: recompute each one from the snapshot with the independent pick
        if n <= 40:
            for i in range(n):
                a = before[i]
                b = before
                dd = D[i, i] + np.diag(D) - D[i, :] - D[:, i]
                ff = F[a, a] + F[b, b] - F[a, b] - F[b, a]
                d = I_before[i, b] + I_before[:, a] - I_before[i, a] - I_before[np.arange(n), b] - dd.astype(np.int64) * ff
                u = oracle.oneshot_uniform(int(_word(oracle, 77, 1, 2, step, i)))
                assert tg[i] == py_pick(oracle, d.astype(np.int64), float(f32(beta)), u)[0]
        moved = np.nonzero(before != phi)[0]
        assert len(moved) == 2 * swaps
        # disjoint transpositions
        for i in moved:
            j = int(np.nonzero(before == phi[i])[0][0])
            assert phi[j] == before[i]
        assert np.array_equal(inv[phi], np.arange(n))
        I_ref, E_ref = oracle.force_init(D, F, phi)
        assert np.array_equal(I, I_ref)
        assert E[0] == E_ref == direct_energy(D.astype(np.int64), F.astype(np.int64), phi)
        assert bestE[0] <= E[0]
    assert total > 0


def _word(oracle, seed, group, replica, step, loc):
    return oracle.lib.orc_sweep_word(seed, group, replica, step, loc, 0)


def test_ballot_rule(oracle):
    """Every applied swap (i, j) is the best ballot at both i and j among the proposals."""
    inst = instances.uniform(30, 2)
    D = np.ascontiguousarray(inst.D, np.int32)
    F = np.ascontiguousarray(inst.F, np.int32)
    phi = np.random.default_rng(1).permutation(30).astype(np.int32)
    inv = np.argsort(phi).astype(np.int32)
    I, E0 = oracle.force_init(D, F, phi)
    E = np.array([E0], np.int64)
    bestE = np.array([2147483647], np.int64)
    for step in range(8):
        before = phi.copy()
        Ib = I.copy()
        _, tg = oracle.oneshot_step(D, F, I, phi, inv, E, bestE, 0.01, 3, 0, 0, step)
        delta = {}
        for i in range(30):
            j = tg[i]
            a, b = before[i], before[j]
            dd = int(D[i, i]) + int(D[j, j]) - int(D[i, j]) - int(D[j, i])
            ff = int(F[a, a]) + int(F[b, b]) - int(F[a, b]) - int(F[b, a])
            delta[i] = int(Ib[i, b] + Ib[j, a] - Ib[i, a] - Ib[j, b]) - dd * ff
        key = {i: (-delta[i], i) for i in range(30) if tg[i] != i}
        owner = {}
        for i, k in key.items():
            for loc in (i, tg[i]):
                if loc not in owner or k < key[owner[loc]]:
                    owner[loc] = i
        accepted = sorted(i for i in key if owner.get(i) == i and owner.get(tg[i]) == i)
        moved = sorted(np.nonzero(before != phi)[0].tolist())
        assert moved == sorted(set(accepted) | {int(tg[i]) for i in accepted})


def test_run_rule_one_improves(oracle):
    inst = instances.uniform(32, 4)
    st = oracle.setup(inst.D, inst.F, 2, 8, 2, 14.4269504089, 1.5849, 11, rule=1)
    start = int(st.E.min())
    oracle.run(st, inst.D, inst.F, 60)
    assert st.single_best < start
    assert st.accepts > 0
    for t in range(2):
        for l in range(8):
            I_ref, E_ref = oracle.force_init(np.ascontiguousarray(inst.D, np.int32),
                                             np.ascontiguousarray(inst.F, np.int32), st.phi[t, l])
            assert np.array_equal(st.I[t, l], I_ref) and st.E[t, l] == E_ref


def test_oneshot_uniforms_match_the_per_word_draws(oracle):
    u = oracle.oneshot_uniforms(123, 6, 3, 5, 7)
    ref = [[oracle.oneshot_uniform(oracle.lib.orc_sweep_word(123, k // 3, k % 3, 5, i, 0)) for i in range(7)]
           for k in range(6)]
    assert np.array_equal(u, np.array(ref, np.float32))


def test_reference_oneshot_harness_loads():
    """GPU-CUPIM's one-shot step as built by oracle/build_cupim.sh (the pin of the one-shot
    oracle, tests/test_gpu_cupim_pin.py, runs it on a GPU): it loads without a GPU and exports
    the harness's entry points."""
    import os
    from oracle import REF_DIR, CupimRef
    path = os.path.join(REF_DIR, "libref_cupim.so")
    if not os.path.exists(path):
        pytest.skip("libref_cupim.so not built (the reference source was absent at build time)")
    ref = CupimRef(path)
    for name in ("cupim_open", "cupim_set", "cupim_step", "cupim_get", "cupim_close"):
        assert hasattr(ref.lib, name)
