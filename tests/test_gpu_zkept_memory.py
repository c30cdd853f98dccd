"""Device blocks kept between solves: a solve on a block another solve used before gives the
same results as one on a fresh allocation, and releasing the kept blocks leaves the library
ready for the next solve."""
import numpy as np
import pytest

import instances

pytestmark = pytest.mark.gpu


def _same(x, y):
    assert x["best_energy"] == y["best_energy"] and x["accepts"] == y["accepts"]
    assert np.array_equal(x["best_perm"], y["best_perm"])
    assert np.array_equal(x["final_energies"], y["final_energies"])


def test_solves_on_kept_and_fresh_blocks_agree(gpu):
    small = instances.uniform(37, 61)
    big = instances.uniform(90, 62)
    p_small = gpu.default_params(replicas=4, groups=3, beta_max=0.01, beta_ratio=1.3, max_megaiters=20, seed=3)
    p_big = gpu.default_params(replicas=8, groups=2, beta_max=0.005, beta_ratio=1.2, max_megaiters=10, seed=4)
    gpu.release_kept_memory()
    fresh = gpu.solve(small.F, small.D, p_small)        # fresh block, kept afterwards
    big1 = gpu.solve(big.F, big.D, p_big)                 # needs a larger block: new one, kept
    again = gpu.solve(small.F, small.D, p_small)          # reuses the big block (old contents)
    _same(fresh, again)
    big2 = gpu.solve(big.F, big.D, p_big)
    _same(big1, big2)
    gpu.release_kept_memory()
    gpu.release_kept_memory()                              # nothing left: a no-op
    _same(fresh, gpu.solve(small.F, small.D, p_small))
