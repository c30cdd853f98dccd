"""Seeded synthetic QAP instances and the reference's instance-file format.

The reference reads a whitespace-separated text file: ``n``, then the n x n flow matrix F,
then the n x n distance matrix D (``CPU-PIM/CPU_PIM.cpp:79-107``).  ``write_instance`` and
``read_instance`` use that format unchanged.

The QAPLIB files the reference was run on are not available, so every workload here is a
seeded synthetic instance.  The generators follow the published workload descriptions:

* ``uniform``       symmetric F and D, int32 uniform in [0, 99], zero diagonal
                    (the n = 32 plain case, and the 512-instance batch with n ~ U[20, 150]);
* ``grid256``       n = 256: F symmetric Bernoulli(0.36) 0/1, zero diagonal; D the squared
                    Euclidean distance between the points of a 16 x 16 integer grid plus a
                    symmetric uniform integer perturbation in [0, 3], zero diagonal;
* ``heavy``         F = round(lognormal(mu=2, sigma=1.5)), symmetric, 70 % of the entries
                    zeroed at random, zero diagonal; D = rounded Euclidean distances between
                    uniform random points in a 1000 x 1000 square
                    (the 128-instance batch with n ~ U[100, 256]);
* ``serving_trace`` Poisson arrivals with n ~ U[30, 256], half ``uniform``, half ``heavy``.

Each instance is a function of (generator, n, seed) only.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Iterator, List, Tuple

import numpy as np


@dataclasses.dataclass
class Instance:
    """One QAP instance: F (flow between facilities) and D (distance between locations)."""

    n: int
    F: np.ndarray  # int32 [n, n]
    D: np.ndarray  # int32 [n, n]
    name: str = ""

    def __post_init__(self):
        self.F = np.ascontiguousarray(self.F, dtype=np.int32)
        self.D = np.ascontiguousarray(self.D, dtype=np.int32)
        if self.F.shape != (self.n, self.n) or self.D.shape != (self.n, self.n):
            raise ValueError("F and D must be n x n")


def _symmetric_from_upper(upper: np.ndarray) -> np.ndarray:
    m = np.triu(upper, 1)
    return m + m.T


def uniform(n: int, seed: int, lo: int = 0, hi: int = 99) -> Instance:
    rng = np.random.default_rng(seed)
    F = _symmetric_from_upper(rng.integers(lo, hi + 1, size=(n, n), dtype=np.int64))
    D = _symmetric_from_upper(rng.integers(lo, hi + 1, size=(n, n), dtype=np.int64))
    return Instance(n, F, D, name=f"uniform_n{n}_s{seed}")


def grid256(seed: int, side: int = 16, p: float = 0.36) -> Instance:
    n = side * side
    rng = np.random.default_rng(seed)
    F = _symmetric_from_upper((rng.random((n, n)) < p).astype(np.int64))
    ys, xs = np.divmod(np.arange(n), side)
    d2 = (xs[:, None] - xs[None, :]) ** 2 + (ys[:, None] - ys[None, :]) ** 2
    pert = _symmetric_from_upper(rng.integers(0, 4, size=(n, n), dtype=np.int64))
    D = d2 + pert
    np.fill_diagonal(D, 0)
    return Instance(n, F, D, name=f"grid256_s{seed}")


def clique_flow(seed: int, side: int = 16, active: int = 92) -> Instance:
    """The structure CPU_PIM_tai256c.cpp is written for: n = side^2 locations on a grid
    (squared Euclidean distance plus a symmetric uniform [0, 3] perturbation, zero diagonal) and
    unit flows between every pair of the first `active` facilities, none elsewhere."""
    n = side * side
    rng = np.random.default_rng(seed)
    F = np.zeros((n, n), np.int64)
    F[:active, :active] = 1
    np.fill_diagonal(F, 0)
    ys, xs = np.divmod(np.arange(n), side)
    d2 = (xs[:, None] - xs[None, :]) ** 2 + (ys[:, None] - ys[None, :]) ** 2
    D = d2 + _symmetric_from_upper(rng.integers(0, 4, size=(n, n), dtype=np.int64))
    np.fill_diagonal(D, 0)
    return Instance(n, F, D, name=f"clique{active}_n{n}_s{seed}")


def heavy(n: int, seed: int, mu: float = 2.0, sigma: float = 1.5, zero_frac: float = 0.7,
          square: float = 1000.0) -> Instance:
    rng = np.random.default_rng(seed)
    flows = np.rint(rng.lognormal(mu, sigma, size=(n, n))).astype(np.int64)
    keep = rng.random((n, n)) >= zero_frac
    F = _symmetric_from_upper(np.where(keep, flows, 0))
    pts = rng.random((n, 2)) * square
    diff = pts[:, None, :] - pts[None, :, :]
    D = np.rint(np.sqrt((diff ** 2).sum(-1))).astype(np.int64)
    np.fill_diagonal(D, 0)
    if F.max() > np.iinfo(np.int32).max:
        raise ValueError("flow exceeds int32")
    return Instance(n, F, D, name=f"heavy_n{n}_s{seed}")


def uniform_batch(count: int = 512, n_lo: int = 20, n_hi: int = 150, seed: int = 3) -> List[Instance]:
    """The mixed-size batch: n ~ U[n_lo, n_hi], each instance seeded by seed*1_000_003 + k."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_lo, n_hi + 1, size=count)
    return [uniform(int(n), seed * 1_000_003 + k) for k, n in enumerate(ns)]


def heavy_batch(count: int = 128, n_lo: int = 100, n_hi: int = 256, seed: int = 4) -> List[Instance]:
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_lo, n_hi + 1, size=count)
    return [heavy(int(n), seed * 1_000_003 + k) for k, n in enumerate(ns)]


def serving_trace(rate_hz: float = 200.0, duration_s: float = 60.0, n_lo: int = 30,
                  n_hi: int = 256, seed: int = 5) -> Iterator[Tuple[float, Instance]]:
    """(arrival time in s, instance) pairs of a Poisson arrival process."""
    rng = np.random.default_rng(seed)
    t = 0.0
    k = 0
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t >= duration_s:
            return
        n = int(rng.integers(n_lo, n_hi + 1))
        sub = seed * 1_000_003 + k
        inst = uniform(n, sub) if (k % 2 == 0) else heavy(n, sub)
        yield t, inst
        k += 1


def write_instance(path: str, inst: Instance) -> None:
    """Reference text format: n, blank line, F rows, blank line, D rows."""
    with open(path, "w") as f:
        f.write(f"{inst.n}\n\n")
        for M in (inst.F, inst.D):
            for row in M:
                f.write(" ".join(str(int(v)) for v in row))
                f.write("\n")
            f.write("\n")


def read_instance(path: str) -> Instance:
    with open(path) as f:
        tok = f.read().split()
    n = int(tok[0])
    vals = np.array([int(v) for v in tok[1:1 + 2 * n * n]], dtype=np.int64)
    if vals.size != 2 * n * n:
        raise ValueError(f"{path}: expected {2 * n * n} matrix entries, found {vals.size}")
    return Instance(n, vals[: n * n].reshape(n, n), vals[n * n:].reshape(n, n),
                    name=os.path.basename(path))
