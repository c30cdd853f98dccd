"""Known-answer tests of the oracle's random-word layer (CPU only)."""
import math
import random

import numpy as np


def test_philox4x32_10_known_answers(oracle):
    # Published Philox4x32-10 vectors (Salmon et al., SC'11, Random123 known-answer tests).
    assert [hex(x) for x in oracle.philox([0, 0, 0, 0], [0, 0])] == \
        ["0x6627e8d5", "0xe169c58d", "0xbc57ac4c", "0x9b00dbd8"]
    assert [hex(x) for x in oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)] == \
        ["0x408f276d", "0x41c83b0e", "0xa20bc7c6", "0x6d5451fd"]
    assert [hex(x) for x in oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                                          [0xA4093822, 0x299F31D0])] == \
        ["0xd16cfe09", "0x94fdcceb", "0x5001e420", "0x24126ea1"]


def test_canonical_matches_definition(oracle):
    rng = random.Random(3)
    for _ in range(2000):
        w0, w1 = rng.getrandbits(32), rng.getrandbits(32)
        s = float(w0) + float(w1) * 4294967296.0
        r = s / 18446744073709551616.0
        if r >= 1.0:
            r = math.nextafter(1.0, 0.0)
        assert oracle.canonical(w0, w1) == r
    assert oracle.canonical(0xFFFFFFFF, 0xFFFFFFFF) == math.nextafter(1.0, 0.0)
    assert oracle.canonical(0, 0) == 0.0


def test_initial_perms_are_permutations(oracle):
    for n, T in ((1, 1), (2, 3), (17, 4), (256, 2)):
        p = oracle.initial_perms(n, T, 99)
        for t in range(T):
            assert sorted(p[t].tolist()) == list(range(n))


def test_force_init_identities(oracle):
    import instances
    inst = instances.uniform(23, 4)
    phi = np.random.default_rng(0).permutation(23).astype(np.int32)
    I, E = oracle.force_init(inst.D, inst.F, phi)
    # E = sum_ij D_ij F_phi(i),phi(j) and sum_i I[i][phi(i)] = -2E
    e = int((inst.D.astype(np.int64) * inst.F[np.ix_(phi, phi)]).sum())
    assert E == e
    assert int(I[np.arange(23), phi].sum()) == -2 * E
