"""ctypes access to the oracle (TEST INFRASTRUCTURE ONLY).

* ``Oracle``     - the C restatement of the CPU_PIM hot path (oracle/liboracle.so).
* ``RefHarness`` - the reference's own CPU_PIM.cpp built by oracle/build_ref.sh
                   (oracle/_ref/libref_*.so); present only where the reference source was
                   available at build time.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")

NO_BEST = 2147483647


class _RunState(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("T", C.c_int), ("R", C.c_int), ("cap", C.c_int), ("numitera", C.c_int),
        ("seed", C.c_uint64),
        ("I", C.c_void_p), ("phi", C.c_void_p), ("phiinv", C.c_void_p),
        ("E", C.c_void_p), ("bestE", C.c_void_p), ("beta", C.c_void_p),
        ("order", C.c_void_p), ("time_since_swap", C.c_void_p), ("thread_best", C.c_void_p),
        ("single_best", C.c_int64), ("megaiters_done", C.c_int64), ("accepts", C.c_int64),
        ("target_megaiter", C.c_int64), ("active", C.c_int32), ("rule", C.c_int32),
    ]


class RunState:
    """Numpy-owned arrays behind an orc_run_state."""

    def __init__(self, n: int, T: int, R: int, cap: int, numitera: int, seed: int):
        self.n, self.T, self.R, self.cap, self.numitera, self.seed = n, T, R, cap, numitera, seed
        self.I = np.zeros((T, R, n, n), np.int64)
        self.phi = np.zeros((T, R, n), np.int32)
        self.phiinv = np.zeros((T, R, n), np.int32)
        self.E = np.zeros((T, R), np.int64)
        self.bestE = np.zeros((T, R), np.int64)
        self.beta = np.zeros((T, R), np.float64)
        self.order = np.zeros((T, cap), np.int32)
        self.time_since_swap = np.zeros(T, np.int32)
        self.thread_best = np.zeros(T, np.int64)
        self.c = _RunState(n, T, R, cap, numitera, seed,
                           self.I.ctypes.data, self.phi.ctypes.data, self.phiinv.ctypes.data,
                           self.E.ctypes.data, self.bestE.ctypes.data, self.beta.ctypes.data,
                           self.order.ctypes.data, self.time_since_swap.ctypes.data,
                           self.thread_best.ctypes.data, 0, 0, 0, -1)

    @property
    def single_best(self) -> int:
        return int(self.c.single_best)

    @property
    def accepts(self) -> int:
        return int(self.c.accepts)

    @property
    def target_megaiter(self) -> int:
        return int(self.c.target_megaiter)

    @property
    def megaiters_done(self) -> int:
        return int(self.c.megaiters_done)


class Oracle:
    def __init__(self, path: Optional[str] = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (run make -C oracle)")
        L = self.lib = C.CDLL(path)
        L.orc_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
        L.orc_sweep_word.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int]
        L.orc_sweep_word.restype = C.c_uint32
        L.orc_shuffle_word.argtypes = [C.c_uint64, C.c_uint64]
        L.orc_shuffle_word.restype = C.c_uint32
        L.orc_canonical.argtypes = [C.c_uint32, C.c_uint32]
        L.orc_canonical.restype = C.c_double
        L.orc_initial_perms.argtypes = [C.c_int, C.c_int, C.c_uint64, _i32p]
        L.orc_beta_ladder.argtypes = [C.c_int, C.c_double, C.c_double, _f64p]
        L.orc_force_init.argtypes = [C.c_int, _i32p, _i32p, _i32p, _i64p, _i64p]
        L.orc_update.argtypes = [C.c_int, _i32p, _i32p, _i64p, _i32p, _i32p, _i64p, _i64p,
                                 C.c_double, C.c_int, C.c_uint32, C.c_uint32, C.c_void_p]
        L.orc_update.restype = C.c_int
        L.orc_replica_sweeps.argtypes = [C.c_int, _i32p, _i32p, _i64p, _i32p, _i32p, _i64p, _i64p,
                                         C.c_double, C.c_uint64, C.c_uint32, C.c_uint32,
                                         C.c_uint32, C.c_int, C.c_void_p]
        L.orc_replica_sweeps.restype = C.c_int64
        L.orc_track_exchange.argtypes = [C.c_int, C.c_int, _i64p, _i64p, _f64p, _i32p, _i32p,
                                         _i64p, _i64p]
        L.orc_track_exchange.restype = C.c_int
        L.orc_setup.argtypes = [C.POINTER(_RunState), _i32p, _i32p, C.c_double, C.c_double]
        L.orc_run.argtypes = [C.POINTER(_RunState), _i32p, _i32p, C.c_int64, C.c_int64]
        L.orc_run.restype = C.c_int
        L.orc_replay_sweeps.argtypes = [C.c_int, _i32p, _i32p, _i64p, _i32p, _i32p, _i64p, _i64p,
                                        C.c_double, C.c_int, _f64p, C.c_void_p]
        L.orc_replay_sweeps.restype = C.c_int64
        L.orc_exp2f_neg.argtypes = [C.c_float]
        L.orc_exp2f_neg.restype = C.c_float
        L.orc_oneshot_uniform.argtypes = [C.c_uint32]
        L.orc_oneshot_uniform.restype = C.c_float
        L.orc_oneshot_uniforms.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_uint32, C.c_int, _f32p]
        L.orc_oneshot_pick.argtypes = [C.c_int, _i64p, C.c_float, C.c_float, _i64p]
        L.orc_oneshot_pick.restype = C.c_int
        L.orc_oneshot_step.argtypes = [C.c_int, _i32p, _i32p, _i64p, _i32p, _i32p, _i64p, _i64p,
                                       C.c_double, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                                       C.c_void_p]
        L.orc_oneshot_step.restype = C.c_int

    def philox(self, ctr, key) -> np.ndarray:
        out = np.zeros(4, np.uint32)
        self.lib.orc_philox4x32_10(np.asarray(ctr, np.uint32), np.asarray(key, np.uint32), out)
        return out

    def canonical(self, w0: int, w1: int) -> float:
        return self.lib.orc_canonical(w0, w1)

    def initial_perms(self, n: int, T: int, seed: int) -> np.ndarray:
        out = np.zeros((T, n), np.int32)
        self.lib.orc_initial_perms(n, T, seed, out)
        return out

    def beta_ladder(self, R: int, beta0: float, delta_beta: float) -> np.ndarray:
        out = np.zeros(R, np.float64)
        self.lib.orc_beta_ladder(R, beta0, delta_beta, out)
        return out

    def force_init(self, D: np.ndarray, F: np.ndarray, phi: np.ndarray):
        n = D.shape[0]
        I = np.zeros((n, n), np.int64)
        E = np.zeros(1, np.int64)
        self.lib.orc_force_init(n, np.ascontiguousarray(D, np.int32), np.ascontiguousarray(F, np.int32),
                                np.ascontiguousarray(phi, np.int32), I, E)
        return I, int(E[0])

    def replica_sweeps(self, D, F, I, phi, phiinv, E, bestE, beta, seed, group, replica,
                       sweep0, nsweeps, record_picks=False):
        """Runs in place on the given arrays (I int64 [n,n], phi/phiinv int32 [n],
        E/bestE int64 [1]).  Returns (accepts, picks or None)."""
        n = D.shape[0]
        picks = np.zeros((nsweeps, n), np.int32) if record_picks else None
        acc = self.lib.orc_replica_sweeps(n, D, F, I, phi, phiinv, E, bestE, beta, seed, group,
                                          replica, sweep0, nsweeps,
                                          picks.ctypes.data if record_picks else None)
        return int(acc), picks

    def setup(self, D, F, T, R, numitera, beta0, delta_beta, seed, cap=None, active=0,
              rule=0) -> RunState:
        """active > 0: the clique-flow update of CPU_PIM_tai256c.cpp with that many active
        facilities (orc_update_clique).  rule = 1: GPU-CUPIM's one-shot parallel steps
        (orc_oneshot_step) instead of sequential sweeps."""
        n = D.shape[0]
        st = RunState(n, T, R, cap if cap is not None else R, numitera, seed)
        st.c.active = active
        st.c.rule = rule
        self.lib.orc_setup(C.byref(st.c), np.ascontiguousarray(D, np.int32),
                           np.ascontiguousarray(F, np.int32), beta0, delta_beta)
        return st

    def track_exchange_all(self, st: RunState) -> None:
        """Every group's tracking + exchange step (the start of the next mega-iteration)."""
        sb = np.array([st.c.single_best], np.int64)
        for t in range(st.T):
            tss = st.time_since_swap[t:t + 1].copy()
            tb = st.thread_best[t:t + 1].copy()
            self.lib.orc_track_exchange(st.R, st.cap, np.ascontiguousarray(st.E[t]),
                                        np.ascontiguousarray(st.bestE[t]), st.beta[t], st.order[t],
                                        tss, tb, sb)
            st.time_since_swap[t] = tss[0]
            st.thread_best[t] = tb[0]
        st.c.single_best = int(sb[0])

    def replay_sweeps(self, D, F, phi, beta, r):
        """Sweeps of one replica from permutation phi with the uniforms r ([nsweeps, n]).
        Returns (phi, I, E, bestE, accepts)."""
        D = np.ascontiguousarray(D, np.int32)
        F = np.ascontiguousarray(F, np.int32)
        phi = np.ascontiguousarray(phi, np.int32).copy()
        inv = np.argsort(phi).astype(np.int32)
        I, E0 = self.force_init(D, F, phi)
        E = np.array([E0], np.int64)
        bestE = np.array([NO_BEST], np.int64)
        r = np.ascontiguousarray(r, np.float64)
        acc = self.lib.orc_replay_sweeps(D.shape[0], D, F, I, phi, inv, E, bestE, beta, r.shape[0], r.ravel(), None)
        return phi, I, int(E[0]), int(bestE[0]), int(acc)

    def exp2f_neg(self, x: float) -> float:
        return float(self.lib.orc_exp2f_neg(x))

    def oneshot_uniform(self, w0: int) -> float:
        return float(self.lib.orc_oneshot_uniform(w0))

    def oneshot_uniforms(self, seed: int, count: int, R: int, step: int, n: int) -> np.ndarray:
        """[count, n] thresholds of one step; replica k is replica k % R of group k // R."""
        out = np.zeros((count, n), np.float32)
        self.lib.orc_oneshot_uniforms(seed, count, R, step, n, out)
        return out

    def oneshot_pick(self, d: np.ndarray, beta_f: float, u: float):
        """(target, delta) of one proposal from the deltas d of every partner location."""
        out = np.zeros(1, np.int64)
        j = self.lib.orc_oneshot_pick(len(d), np.ascontiguousarray(d, np.int64), beta_f, u, out)
        return int(j), int(out[0])

    def oneshot_step(self, D, F, I, phi, phiinv, E, bestE, beta, seed, group, replica, step):
        """One one-shot step in place (I int64 [n,n], phi/phiinv int32 [n], E/bestE int64 [1]).
        Returns (swaps applied, every location's proposal)."""
        n = D.shape[0]
        tg = np.zeros(n, np.int32)
        np_ = self.lib.orc_oneshot_step(n, np.ascontiguousarray(D, np.int32), np.ascontiguousarray(F, np.int32),
                                        I, phi, phiinv, E, bestE, beta, seed, group, replica, step,
                                        tg.ctypes.data)
        return int(np_), tg

    def run(self, st: RunState, D, F, megaiters: int, goal: int = 0) -> int:
        return self.lib.orc_run(C.byref(st.c), np.ascontiguousarray(D, np.int32),
                                np.ascontiguousarray(F, np.int32), megaiters, goal)


def ref_available(variant: str = "big") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{variant}.so"))


class RefHarness:
    """The reference's CPU_PIM.cpp, driven through oracle/ref_harness.cpp.  Each variant is
    a separate library with its own copy of the reference's globals."""

    _loaded: Dict[str, "RefHarness"] = {}

    def __new__(cls, variant: str = "big"):
        if variant in cls._loaded:
            return cls._loaded[variant]
        self = super().__new__(cls)
        path = os.path.join(REF_DIR, f"libref_{variant}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (needs the reference source; run make -C oracle)")
        L = self.lib = C.CDLL(path)
        for name in ("ref_maxn", "ref_maxr", "ref_maxt", "ref_has_shim", "ref_n"):
            getattr(L, name).restype = C.c_int
        L.ref_load.argtypes = [C.c_int, _i32p, _i32p]
        L.ref_read_file.argtypes = [C.c_char_p]
        L.ref_get_instance.argtypes = [_i32p, _i32p]
        L.ref_setup.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_uint64]
        L.ref_set_goal.argtypes = [C.c_int]
        L.ref_setup_replicated.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_uint64]
        L.ref_run.argtypes = [C.c_int]
        L.ref_run.restype = C.c_double
        L.ref_domega.argtypes = [C.c_int, C.c_int]
        L.ref_get_replica.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _i64p, _i64p, _i64p, _f64p]
        L.ref_get_group.argtypes = [C.c_int, _i32p, _i32p, _i64p]
        L.ref_single_best.restype = C.c_int64
        L.ref_quiet.argtypes = [C.c_int]
        L.ref_quiet(1)
        self.maxn, self.maxr, self.maxt = L.ref_maxn(), L.ref_maxr(), L.ref_maxt()
        self.has_shim = bool(L.ref_has_shim())
        self.variant = variant
        cls._loaded[variant] = self
        return self

    def load(self, F: np.ndarray, D: np.ndarray) -> None:
        n = F.shape[0]
        if self.lib.ref_load(n, np.ascontiguousarray(F, np.int32), np.ascontiguousarray(D, np.int32)):
            raise ValueError(f"n={n} exceeds the reference's MAXN={self.maxn}")

    def read_file(self, path: str) -> int:
        return self.lib.ref_read_file(path.encode())

    def instance(self):
        n = self.lib.ref_n()
        F = np.zeros((n, n), np.int32)
        D = np.zeros((n, n), np.int32)
        self.lib.ref_get_instance(F, D)
        return F, D

    def setup(self, T, R, numitera, beta0, delta_beta, seed) -> None:
        if self.lib.ref_setup(T, R, numitera, beta0, delta_beta, seed):
            raise ValueError("reference setup rejected the parameters")
        self.T, self.R = T, R

    def setup_replicated(self, T, R, numitera, beta0, delta_beta, seed) -> None:
        """Group 0 by the reference's setup(), the other groups as copies (timing only)."""
        if self.lib.ref_setup_replicated(T, R, numitera, beta0, delta_beta, seed):
            raise ValueError("reference setup rejected the parameters")
        self.T, self.R = T, R

    def run(self, megaiters: int) -> float:
        """megaiters iterations of threadToRun on one thread per group; wall seconds."""
        return self.lib.ref_run(megaiters)

    def replica(self, t: int, l: int):
        n = self.lib.ref_n()
        phi = np.zeros(n, np.int32)
        inv = np.zeros(n, np.int32)
        I = np.zeros((n, n), np.int64)
        E = np.zeros(1, np.int64)
        bE = np.zeros(1, np.int64)
        b = np.zeros(1, np.float64)
        self.lib.ref_get_replica(t, l, phi, inv, I, E, bE, b)
        return dict(phi=phi, phiinv=inv, I=I, E=int(E[0]), bestE=int(bE[0]), beta=float(b[0]))

    def group(self, t: int):
        order = np.zeros(self.maxr, np.int32)
        tss = np.zeros(1, np.int32)
        tb = np.zeros(1, np.int64)
        self.lib.ref_get_group(t, order, tss, tb)
        return dict(order=order, time_since_swap=int(tss[0]), thread_best=int(tb[0]))

    def single_best(self) -> int:
        return int(self.lib.ref_single_best())


class CupimRef:
    """GPU-CUPIM's own one-shot step (perl-gpu/src/lib/qap/qap.cu:1462-1600) built by
    oracle/build_cupim.sh into _ref/libref_cupim.so and driven through oracle/cupim_harness.cu:
    one pool of R replicas (float betas, int32 force matrices) whose step consumes the
    thresholds the caller uploads.  Needs a GPU; one pool per process at a time."""

    def __init__(self, path: Optional[str] = None):
        path = path or os.path.join(REF_DIR, "libref_cupim.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (needs the reference source; run make -C oracle)")
        L = self.lib = C.CDLL(path)
        L.cupim_open.argtypes = [C.c_char_p, C.c_int]
        L.cupim_set.argtypes = [_i32p, _f32p]
        L.cupim_step.argtypes = [_f32p]
        L.cupim_get.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        for f in (L.cupim_open, L.cupim_set, L.cupim_step, L.cupim_get, L.cupim_close):
            f.restype = C.c_int
        self.n = self.R = 0

    @staticmethod
    def _ok(rc: int, what: str) -> None:
        if rc != 0:
            raise RuntimeError(f"{what} failed: {rc}")

    def open(self, path: str, R: int) -> None:
        """A pool of R replicas on the instance file at path (n, then F, then D)."""
        self._ok(self.lib.cupim_open(path.encode(), R), "cupim_open")
        with open(path) as f:
            self.n = int(f.readline().split()[0])
        self.R = R

    def set(self, phi: np.ndarray, betas: np.ndarray) -> None:
        """Every replica's permutation [R, n] and beta (binary32); the reference recomputes the
        force matrices and energies."""
        self._ok(self.lib.cupim_set(np.ascontiguousarray(phi, np.int32), np.ascontiguousarray(betas, np.float32)),
                 "cupim_set")

    def step(self, u: np.ndarray) -> None:
        """One step of every replica with the thresholds u [R, n]."""
        self._ok(self.lib.cupim_step(np.ascontiguousarray(u, np.float32)), "cupim_step")

    def get(self, force: bool = True):
        """(phi [R, n], force [R, n, n] or None, energy [R], resolved proposals [R, n])."""
        R, n = self.R, self.n
        phi = np.zeros((R, n), np.int32)
        frc = np.zeros((R, n, n), np.int32) if force else None
        score = np.zeros(R, np.int32)
        tg = np.zeros((R, n), np.int32)
        self._ok(self.lib.cupim_get(phi.ctypes.data, frc.ctypes.data if force else None, score.ctypes.data,
                                    tg.ctypes.data), "cupim_get")
        return phi, frc, score, tg

    def close(self) -> None:
        self._ok(self.lib.cupim_close(), "cupim_close")
