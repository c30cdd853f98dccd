"""Shared test setup: the gpu marker and import paths.

CPU tests (-m "not gpu") pin the oracle to the reference and check the host logic; GPU tests
(-m gpu) compare the CUDA solver, called through its C ABI, with the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "p-dit-probabilistic-ising-machine-for-solving-the-quadratic-assignment-problem_b200")
for p in (PKG, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built CUDA library")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def gpu():
    """The solver binding; fails (not skips) when a GPU test runs without the library or GPU."""
    import pimqap
    if not _has_gpu():
        pytest.fail("GPU test selected but no CUDA device is visible")
    pimqap.lib()
    return pimqap
