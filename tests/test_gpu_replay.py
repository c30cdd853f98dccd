"""pimqap_sweep_replay and the asynchronous batch API on the GPU.

The replay runs one replica's sweeps with the uniforms the caller gives.  Here they come from
an MT19937 word stream (numpy's legacy seeding, the generator std::mt19937(seed) produces)
combined as generate_canonical<double, 53> combines two words, i.e. the kind of stream the
reference itself draws (CPU_PIM.cpp:212) rather than this project's Philox stream.  The GPU
must then reproduce the oracle's sweeps bit for bit: permutation, force matrix, energy, best
energy, accepted moves.
"""
import numpy as np
import pytest

import instances
from test_gpu_parity import asym, binary

pytestmark = pytest.mark.gpu


def mt_uniforms(seed, count):
    """count doubles (w0 + w1 * 2^32) * 2^-64 from consecutive MT19937 words, as
    std::generate_canonical<double, 53> forms them from std::mt19937(seed)."""
    bg = np.random.MT19937()
    bg._legacy_seeding(seed)
    w = bg.random_raw(2 * count).astype(np.uint64)
    s = (w[0::2].astype(np.float64) + w[1::2].astype(np.float64) * 4294967296.0)
    r = s * 2.0 ** -64
    return np.minimum(r, np.nextafter(1.0, 0.0))


# name: (instance, beta (internal), sweeps, extra params)
CASES = {
    "grid256_binary_kernel": (lambda: instances.grid256(41), 0.03125, 3, {}),
    "grid256_generic_kernel": (lambda: instances.grid256(41), 0.03125, 2, {"compact_instance": 1}),
    "uniform_n40": (lambda: instances.uniform(40, 42), 0.002, 6, {}),
    "asym_n30_cluster2": (lambda: asym(30, 43), 0.01, 5, {"cluster_size": 2}),
    "binary_n70_cluster4": (lambda: binary(70, 44), 0.02, 4, {"cluster_size": 4}),
    "uniform_n24_int64": (lambda: instances.uniform(24, 45), 0.005, 8, {"force_bits": 64}),
}


@pytest.mark.parametrize("name", list(CASES))
def test_replay_matches_oracle_on_an_mt19937_stream(gpu, oracle, name):
    make, beta, sweeps, extra = CASES[name]
    inst = make()
    n = inst.n
    rng = np.random.default_rng(n + sweeps)
    phi = rng.permutation(n).astype(np.int32)
    r = mt_uniforms(5489 + n, sweeps * n).reshape(sweeps, n)
    p = gpu.default_params(beta_max=beta, beta_internal=1, **extra)
    got = gpu.sweep_replay(inst.F, inst.D, p, phi, r)
    o_phi, o_I, o_E, o_bE, o_acc = oracle.replay_sweeps(inst.D, inst.F, phi, beta, r)
    assert np.array_equal(got["phi"], o_phi)
    assert np.array_equal(got["I"], o_I)
    assert (got["E"], got["bestE"], got["accepts"]) == (o_E, o_bE, o_acc)
    assert o_acc > 0


def test_replay_zero_sweeps_is_the_set_up(gpu, oracle):
    inst = instances.uniform(17, 46)
    phi = np.random.default_rng(1).permutation(17).astype(np.int32)
    got = gpu.sweep_replay(inst.F, inst.D, gpu.default_params(beta_max=0.1), phi, np.zeros((0, 17)))
    I, E = oracle.force_init(np.ascontiguousarray(inst.D, np.int32), np.ascontiguousarray(inst.F, np.int32), phi)
    assert np.array_equal(got["phi"], phi) and np.array_equal(got["I"], I) and got["E"] == E
    assert got["accepts"] == 0


def test_async_batch_equals_synchronous_batch(gpu):
    insts = [instances.uniform(n, 50 + n) for n in (23, 37, 61)]
    params = [gpu.default_params(replicas=4, groups=2, beta_max=0.01, beta_ratio=1.3, max_megaiters=30,
                                 seed=7 + k) for k in range(3)]
    sync = gpu.batch_solve([(i.F, i.D) for i in insts], params)
    b = gpu.Batch([(i.F, i.D) for i in insts], params)
    res = b.wait(120.0)
    assert res is not None and b.poll()
    b.close()
    for x, y in zip(sync, res):
        assert x["best_energy"] == y["best_energy"] and x["accepts"] == y["accepts"]
        assert np.array_equal(x["best_perm"], y["best_perm"])
        assert np.array_equal(x["final_energies"], y["final_energies"])
