"""Python binding of the solver's C ABI (``include/pimqap.h``) over ctypes.

The solver itself is ``csrc/libpimqap.so`` (host runtime + sm_100a kernels).  This module
only marshals arguments; it has no compute path of its own, and every call fails loudly
when the library is missing or has no usable GPU.

Reference mapping (``CPU-PIM/CPU_PIM.cpp``): ``read_problem`` is readProblem() (:79-107),
``Solver`` is setup() + the threadToRun() loop (:109-364), ``solve`` is main() (:612-684).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "csrc", "libpimqap.so")

OK = 0
NOT_READY = 8
STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_IO", 3: "ERR_CUDA", 4: "ERR_NO_DEVICE", 5: "ERR_RANGE",
          6: "ERR_DEVICE", 7: "ERR_BUSY", 8: "ERR_NOT_READY"}
NO_BEST = 2147483647
MAX_N = 256
MAX_REPLICAS = 64
LN2_INV = 1.44269504089  # the reference's -b scaling (CPU_PIM.cpp:528)


class PimqapError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Instance(C.Structure):
    _fields_ = [("n", C.c_int32), ("flow", C.POINTER(C.c_int32)), ("dist", C.POINTER(C.c_int32))]


class ClassTuning(C.Structure):
    _fields_ = [("force_bits", C.c_int32), ("cluster_size", C.c_int32), ("band", C.c_int32),
                ("n_max", C.c_int32), ("members", C.c_int32), ("threads", C.c_int32),
                ("workers", C.c_int32), ("grid", C.c_int32), ("fixed_threads", C.c_int32),
                ("fixed_workers", C.c_int32), ("tried", C.c_int32), ("pad", C.c_int32),
                ("fixed_ms", C.c_double), ("tuned_ms", C.c_double)]


class Params(C.Structure):
    _fields_ = [
        ("replicas", C.c_int32), ("groups", C.c_int32), ("sweeps_per_exchange", C.c_int32),
        ("rank_slots", C.c_int32), ("max_megaiters", C.c_int64), ("beta_max", C.c_double),
        ("beta_ratio", C.c_double), ("goal", C.c_int64), ("timeout_s", C.c_double),
        ("seed", C.c_uint64), ("force_bits", C.c_int32), ("device", C.c_int32),
        ("megaiters_per_launch", C.c_int32), ("threads_per_block", C.c_int32),
        ("cluster_size", C.c_int32), ("beta_internal", C.c_int32), ("auto_beta", C.c_int32),
        ("auto_lower", C.c_double), ("auto_higher", C.c_double), ("goal_print", C.c_int64),
        ("event_capacity", C.c_int32), ("event_perm_capacity", C.c_int32),
        ("compact_instance", C.c_int32), ("active_facilities", C.c_int32),
        ("update_rule", C.c_int32),
        ("replica_pairing", C.c_int32),
        ("launch_mode", C.c_int32),
        ("sweep_pipeline", C.c_int32),
        ("tensor_update", C.c_int32),
        ("oneshot_weights", C.c_int32),
    ]


RULE_SEQUENTIAL = 0
RULE_ONE_SHOT = 1


EVENT_GROUP_BEST = 0
EVENT_GOAL_PRINT = 1
AUTO_STEPS = 32
AUTO_TRIALS = 5


class Event(C.Structure):
    _fields_ = [("megaiter", C.c_int64), ("energy", C.c_int64), ("time_ms", C.c_double),
                ("kind", C.c_int32), ("group", C.c_int32), ("replica", C.c_int32),
                ("perm_index", C.c_int32), ("trial", C.c_int32), ("pad", C.c_int32)]


class AutoReport(C.Structure):
    _fields_ = [("beta0_internal", C.c_double), ("delta_beta", C.c_double),
                ("min_beta", C.c_double), ("max_beta", C.c_double),
                ("min_beta_printed", C.c_int32), ("pad0", C.c_int32),
                ("avg_energy", C.c_double * AUTO_STEPS),
                ("trial_best", C.c_int64 * (AUTO_STEPS * AUTO_TRIALS)),
                ("steps_printed", C.c_int32), ("goal_trial", C.c_int32),
                ("best_energy", C.c_int64), ("best_perm", C.POINTER(C.c_int32)),
                ("events", C.POINTER(Event)), ("event_capacity", C.c_int32),
                ("event_count", C.c_int32), ("events_dropped", C.c_int64), ("device_ms", C.c_double)]


class Result(C.Structure):
    _fields_ = [
        ("best_energy", C.c_int64), ("best_perm", C.POINTER(C.c_int32)),
        ("target_megaiter", C.c_int64), ("time_to_target_ms", C.c_double),
        ("megaiters_done", C.c_int64), ("updates", C.c_int64), ("accepts", C.c_int64),
        ("device_ms", C.c_double), ("wall_ms", C.c_double), ("force_bits", C.c_int32),
        ("cluster_size", C.c_int32), ("stopped_by", C.c_int32), ("launches", C.c_int32),
        ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64),
        ("final_energies", C.POINTER(C.c_int64)), ("beta_max_used", C.c_double),
        ("beta_ratio_used", C.c_double), ("admit_ms", C.c_double), ("latency_ms", C.c_double),
        ("sweeps", C.c_int64), ("proposals", C.c_int64),
    ]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("memory_budget_bytes", C.c_int64), ("slots_per_class", C.c_int32),
                ("heartbeat_timeout_s", C.c_double), ("sample", C.POINTER(Instance)),
                ("sample_params", C.POINTER(Params)), ("sample_count", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("admitted", C.c_int64), ("completed", C.c_int64),
                ("pending", C.c_int64), ("memory_in_use", C.c_int64), ("memory_budget", C.c_int64),
                ("classes", C.c_int32), ("error_word", C.c_int32)]


_lib = None


def lib() -> C.CDLL:
    """Loads csrc/libpimqap.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is not built (run make -C csrc or __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    st = C.c_int
    L.pimqap_default_params.argtypes = [C.POINTER(Params)]
    L.pimqap_default_params.restype = None
    L.pimqap_last_error.restype = C.c_char_p
    L.pimqap_version.restype = C.c_char_p
    L.pimqap_read_problem.argtypes = [C.c_char_p, C.c_int32, C.POINTER(C.c_int32), C.c_void_p, C.c_void_p]
    L.pimqap_read_problem.restype = st
    L.pimqap_solve.argtypes = [C.POINTER(Instance), C.POINTER(Params), C.POINTER(Result)]
    L.pimqap_solve.restype = st
    L.pimqap_solver_create.argtypes = [C.POINTER(Instance), C.POINTER(Params), C.POINTER(C.c_void_p)]
    L.pimqap_solver_create.restype = st
    L.pimqap_solver_run.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_double)]
    L.pimqap_solver_run.restype = st
    L.pimqap_solver_result.argtypes = [C.c_void_p, C.POINTER(Result)]
    L.pimqap_solver_result.restype = st
    L.pimqap_solver_replica.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p]
    L.pimqap_solver_replica.restype = st
    L.pimqap_solver_group.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    L.pimqap_solver_group.restype = st
    L.pimqap_solver_destroy.argtypes = [C.c_void_p]
    L.pimqap_solver_destroy.restype = None
    L.pimqap_release_kept_memory.argtypes = []
    L.pimqap_release_kept_memory.restype = st
    L.pimqap_batch_solve.argtypes = [C.POINTER(Instance), C.POINTER(Params), C.c_int32, C.POINTER(Result)]
    L.pimqap_batch_solve.restype = st
    L.pimqap_batch_tune.argtypes = [C.POINTER(Instance), C.POINTER(Params), C.c_int32, C.POINTER(ClassTuning),
                                    C.c_int32, C.POINTER(C.c_int32)]
    L.pimqap_batch_tune.restype = st
    L.pimqap_server_create.argtypes = [C.POINTER(ServerConfig), C.POINTER(C.c_void_p)]
    L.pimqap_server_create.restype = st
    L.pimqap_server_submit.argtypes = [C.c_void_p, C.POINTER(Instance), C.POINTER(Params), C.POINTER(C.c_int64)]
    L.pimqap_server_submit.restype = st
    L.pimqap_server_poll.argtypes = [C.c_void_p, C.c_int64, C.POINTER(Result)]
    L.pimqap_server_poll.restype = st
    L.pimqap_server_wait.argtypes = [C.c_void_p, C.c_int64, C.c_double, C.POINTER(Result)]
    L.pimqap_server_wait.restype = st
    L.pimqap_server_stats_get.argtypes = [C.c_void_p, C.POINTER(ServerStats)]
    L.pimqap_server_stats_get.restype = st
    L.pimqap_server_destroy.argtypes = [C.c_void_p]
    L.pimqap_server_destroy.restype = None
    L.pimqap_server_debug_stall_heartbeat.argtypes = [C.c_void_p, C.c_int32]
    L.pimqap_server_debug_stall_heartbeat.restype = None
    L.pimqap_auto_beta.argtypes = [C.POINTER(Instance), C.POINTER(Params), C.POINTER(C.c_double),
                                   C.POINTER(C.c_double), C.c_void_p, C.POINTER(C.c_int64), C.c_void_p]
    L.pimqap_auto_beta.restype = st
    L.pimqap_solver_events.argtypes = [C.c_void_p, C.c_int64, C.c_int32, C.POINTER(Event),
                                       C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.pimqap_solver_events.restype = st
    L.pimqap_solver_event_perm.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
    L.pimqap_solver_event_perm.restype = st
    L.pimqap_auto_beta_report.argtypes = [C.POINTER(Instance), C.POINTER(Params), C.POINTER(AutoReport)]
    L.pimqap_auto_beta_report.restype = st
    L.pimqap_solve_static.argtypes = [C.POINTER(Instance), C.POINTER(Params), C.POINTER(Result)]
    L.pimqap_solve_static.restype = st
    L.pimqap_probe_smem_bandwidth.argtypes = [C.c_int32, C.POINTER(C.c_double)]
    L.pimqap_probe_smem_bandwidth.restype = st
    L.pimqap_probe_weight_exp2.argtypes = [C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int64]
    L.pimqap_probe_weight_exp2.restype = st
    L.pimqap_load_file.argtypes = [C.c_char_p, C.POINTER(Instance)]
    L.pimqap_load_file.restype = st
    L.pimqap_free_instance.argtypes = [C.POINTER(Instance)]
    L.pimqap_free_instance.restype = None
    L.pimqap_sweep_replay.argtypes = [C.POINTER(Instance), C.POINTER(Params), C.c_void_p, C.c_int32,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.pimqap_sweep_replay.restype = st
    L.pimqap_batch_submit.argtypes = [C.POINTER(Instance), C.POINTER(Params), C.c_int32, C.POINTER(Result),
                                      C.POINTER(C.c_void_p)]
    L.pimqap_batch_submit.restype = st
    L.pimqap_batch_poll.argtypes = [C.c_void_p]
    L.pimqap_batch_poll.restype = st
    L.pimqap_batch_wait.argtypes = [C.c_void_p, C.c_double]
    L.pimqap_batch_wait.restype = st
    L.pimqap_batch_release.argtypes = [C.c_void_p]
    L.pimqap_batch_release.restype = None
    _lib = L
    return L


def _check(status: int) -> None:
    if status != OK:
        raise PimqapError(status, lib().pimqap_last_error().decode(errors="replace"))


def default_params(**kw) -> Params:
    p = Params()
    lib().pimqap_default_params(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


class _Inst:
    """Keeps the numpy buffers of a pimqap_instance alive."""

    def __init__(self, F: np.ndarray, D: np.ndarray):
        self.F = np.ascontiguousarray(F, dtype=np.int32)
        self.D = np.ascontiguousarray(D, dtype=np.int32)
        n = self.F.shape[0]
        if self.F.shape != (n, n) or self.D.shape != (n, n):
            raise ValueError("flow and dist must be n x n")
        self.c = Instance(n, self.F.ctypes.data_as(C.POINTER(C.c_int32)),
                          self.D.ctypes.data_as(C.POINTER(C.c_int32)))


def load_file(path: str):
    """pimqap_load_file: (F, D) as int32 arrays, read into library-allocated memory and copied."""
    inst = Instance()
    _check(lib().pimqap_load_file(path.encode(), C.byref(inst)))
    try:
        n = inst.n
        F = np.ctypeslib.as_array(inst.flow, shape=(n, n)).copy()
        D = np.ctypeslib.as_array(inst.dist, shape=(n, n)).copy()
    finally:
        lib().pimqap_free_instance(C.byref(inst))
    return F, D


def sweep_replay(F: np.ndarray, D: np.ndarray, params: Params, phi: np.ndarray, r: np.ndarray) -> dict:
    """nsweeps sweeps of one replica from phi with the uniforms r ([nsweeps, n])."""
    inst = _Inst(F, D)
    n = inst.F.shape[0]
    r = np.ascontiguousarray(r, np.float64).reshape(-1, n)
    phi = np.ascontiguousarray(phi, np.int32)
    out_phi = np.zeros(n, np.int32)
    force = np.zeros((n, n), np.int64)
    E = np.zeros(1, np.int64)
    bE = np.zeros(1, np.int64)
    acc = np.zeros(1, np.int64)
    _check(lib().pimqap_sweep_replay(C.byref(inst.c), C.byref(params), phi.ctypes.data, r.shape[0],
                                     r.ctypes.data, out_phi.ctypes.data, force.ctypes.data, E.ctypes.data,
                                     bE.ctypes.data, acc.ctypes.data))
    return dict(phi=out_phi, I=force, E=int(E[0]), bestE=int(bE[0]), accepts=int(acc[0]))


class Batch:
    """pimqap_batch_submit / poll / wait / release: a batch that runs while the caller goes on."""

    def __init__(self, instances: Sequence, params: Sequence[Params]):
        self._keep = [_Inst(F, D) for F, D in instances]
        count = len(self._keep)
        insts = (Instance * count)(*[k.c for k in self._keep])
        ps = (Params * count)(*params)
        self._perms = [np.zeros(k.F.shape[0], np.int32) for k in self._keep]
        self._energies = [np.zeros(max(1, p.groups * p.replicas), np.int64) for p in params]
        self._rs = (Result * count)()
        for r, p, e in zip(self._rs, self._perms, self._energies):
            r.best_perm = p.ctypes.data_as(C.POINTER(C.c_int32))
            r.final_energies = e.ctypes.data_as(C.POINTER(C.c_int64))
        self._h = C.c_void_p()
        _check(lib().pimqap_batch_submit(insts, ps, count, self._rs, C.byref(self._h)))

    def poll(self) -> bool:
        st = lib().pimqap_batch_poll(self._h)
        if st == NOT_READY:
            return False
        _check(st)
        return True

    def wait(self, timeout: float = -1.0) -> Optional[List[dict]]:
        """The results, or None when timeout (s) ran out first (< 0: no limit)."""
        st = lib().pimqap_batch_wait(self._h, timeout)
        if st == NOT_READY:
            return None
        _check(st)
        return [_result_dict(r, p, e) for r, p, e in zip(self._rs, self._perms, self._energies)]

    def close(self) -> None:
        if self._h:
            lib().pimqap_batch_release(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_problem(path: str, max_n: int = MAX_N):
    """The reference's file reader: returns (F, D) as int32 arrays."""
    n = C.c_int32(0)
    _check(lib().pimqap_read_problem(path.encode(), max_n, C.byref(n), None, None))
    F = np.zeros((n.value, n.value), np.int32)
    D = np.zeros((n.value, n.value), np.int32)
    _check(lib().pimqap_read_problem(path.encode(), max_n, C.byref(n), F.ctypes.data, D.ctypes.data))
    return F, D


def _result_dict(r: Result, perm: Optional[np.ndarray], energies: Optional[np.ndarray] = None) -> dict:
    d = {k: getattr(r, k) for k, _ in Result._fields_ if k not in ("best_perm", "final_energies")}
    d["best_perm"] = perm
    d["final_energies"] = energies
    return d


def _new_result(n: int, replicas_total: int):
    perm = np.zeros(n, np.int32)
    energies = np.zeros(max(1, replicas_total), np.int64)
    r = Result()
    r.best_perm = perm.ctypes.data_as(C.POINTER(C.c_int32))
    r.final_energies = energies.ctypes.data_as(C.POINTER(C.c_int64))
    return r, perm, energies


def solve(F: np.ndarray, D: np.ndarray, params: Params) -> dict:
    inst = _Inst(F, D)
    r, perm, energies = _new_result(inst.F.shape[0], params.groups * params.replicas)
    _check(lib().pimqap_solve(C.byref(inst.c), C.byref(params), C.byref(r)))
    return _result_dict(r, perm, energies)


def release_kept_memory() -> None:
    """pimqap_release_kept_memory: frees the device blocks finished solves left for reuse."""
    _check(lib().pimqap_release_kept_memory())


def auto_beta(F: np.ndarray, D: np.ndarray, params: Params) -> dict:
    """The reference's automatic beta selection; returns beta0 (internal units), deltaBeta,
    the 32 average energies and the best energy / permutation of the trials."""
    inst = _Inst(F, D)
    b0 = C.c_double(0)
    db = C.c_double(0)
    avg = np.zeros(32, np.float64)
    best = C.c_int64(0)
    perm = np.zeros(inst.F.shape[0], np.int32)
    _check(lib().pimqap_auto_beta(C.byref(inst.c), C.byref(params), C.byref(b0), C.byref(db),
                                  avg.ctypes.data, C.byref(best), perm.ctypes.data))
    return dict(beta0=b0.value, delta_beta=db.value, avg_energy=avg, best_energy=best.value,
                best_perm=perm)


def _event_dict(e: Event) -> dict:
    return dict(megaiter=int(e.megaiter), energy=int(e.energy), time_ms=float(e.time_ms),
                kind=int(e.kind), group=int(e.group), replica=int(e.replica),
                perm_index=int(e.perm_index), trial=int(e.trial))


def auto_beta_report(F: np.ndarray, D: np.ndarray, params: Params, event_capacity: int = 1 << 16) -> dict:
    """pimqap_auto_beta_report: everything automatic mode prints and decides."""
    inst = _Inst(F, D)
    rep = AutoReport()
    perm = np.zeros(inst.F.shape[0], np.int32)
    evs = (Event * max(1, event_capacity))()
    rep.best_perm = perm.ctypes.data_as(C.POINTER(C.c_int32))
    rep.events = evs
    rep.event_capacity = event_capacity
    _check(lib().pimqap_auto_beta_report(C.byref(inst.c), C.byref(params), C.byref(rep)))
    return dict(beta0=rep.beta0_internal, delta_beta=rep.delta_beta, min_beta=rep.min_beta,
                max_beta=rep.max_beta, min_beta_printed=bool(rep.min_beta_printed),
                avg_energy=np.array(rep.avg_energy[:]),
                trial_best=np.array(rep.trial_best[:], np.int64), steps_printed=rep.steps_printed,
                goal_trial=rep.goal_trial, best_energy=rep.best_energy, best_perm=perm,
                events=[_event_dict(evs[k]) for k in range(rep.event_count)],
                events_dropped=rep.events_dropped, device_ms=rep.device_ms)


def solve_static(F: np.ndarray, D: np.ndarray, params: Params) -> dict:
    """pimqap_solve_static: the same solve with no device allocation (fixed 8 MiB scratch)."""
    inst = _Inst(F, D)
    perm = np.zeros(inst.F.shape[0], np.int32)
    r = Result()
    r.best_perm = perm.ctypes.data_as(C.POINTER(C.c_int32))
    _check(lib().pimqap_solve_static(C.byref(inst.c), C.byref(params), C.byref(r)))
    return _result_dict(r, perm)


def batch_tune(instances: Sequence, params: Sequence[Params]) -> List[dict]:
    """pimqap_batch_tune: the autotuner's class shapes for this batch (timing them if new)."""
    keep = [_Inst(F, D) for F, D in instances]
    count = len(keep)
    insts = (Instance * count)(*[k.c for k in keep])
    ps = (Params * count)(*params)
    out = (ClassTuning * 64)()
    n = C.c_int32(0)
    _check(lib().pimqap_batch_tune(insts, ps, count, out, 64, C.byref(n)))
    return [{k: getattr(out[i], k) for k, _ in ClassTuning._fields_ if k != "pad"} for i in range(min(n.value, 64))]


def batch_solve(instances: Sequence, params: Sequence[Params]) -> List[dict]:
    """instances: sequence of (F, D); params: one Params per instance."""
    keep = [_Inst(F, D) for F, D in instances]
    count = len(keep)
    insts = (Instance * count)(*[k.c for k in keep])
    ps = (Params * count)(*params)
    perms = [np.zeros(k.F.shape[0], np.int32) for k in keep]
    energies = [np.zeros(max(1, p.groups * p.replicas), np.int64) for p in params]
    rs = (Result * count)()
    for r, p, e in zip(rs, perms, energies):
        r.best_perm = p.ctypes.data_as(C.POINTER(C.c_int32))
        r.final_energies = e.ctypes.data_as(C.POINTER(C.c_int64))
    _check(lib().pimqap_batch_solve(insts, ps, count, rs))
    return [_result_dict(r, p, e) for r, p, e in zip(rs, perms, energies)]


def probe_weight_exp2(x: np.ndarray, device: int = 0) -> np.ndarray:
    """The one-shot rule's binary32 weight function 2^x (x <= 0), evaluated by the device code."""
    xs = np.ascontiguousarray(x, np.float32)
    ys = np.zeros_like(xs)
    fp = C.POINTER(C.c_float)
    _check(lib().pimqap_probe_weight_exp2(device, xs.ctypes.data_as(fp), ys.ctypes.data_as(fp), xs.size))
    return ys


def probe_smem_bandwidth(device: int = 0) -> float:
    """Measured shared-memory read-modify-write bandwidth of the device, GB/s."""
    v = C.c_double(0)
    _check(lib().pimqap_probe_smem_bandwidth(device, C.byref(v)))
    return v.value


class Solver:
    """A solver handle: setup() on construction, then run() mega-iterations at a time."""

    def __init__(self, F: np.ndarray, D: np.ndarray, params: Params):
        self._inst = _Inst(F, D)
        self.params = params
        self.n = self._inst.F.shape[0]
        h = C.c_void_p()
        _check(lib().pimqap_solver_create(C.byref(self._inst.c), C.byref(params), C.byref(h)))
        self.h = h

    def run(self, megaiters: int) -> float:
        """Runs megaiters mega-iterations; returns their device time in ms."""
        ms = C.c_double(0)
        _check(lib().pimqap_solver_run(self.h, megaiters, C.byref(ms)))
        return ms.value

    def result(self) -> dict:
        r, perm, energies = _new_result(self.n, self.params.groups * self.params.replicas)
        _check(lib().pimqap_solver_result(self.h, C.byref(r)))
        return _result_dict(r, perm, energies)

    def replica(self, t: int, l: int, force: bool = True) -> dict:
        """State of replica l of group t; force=False skips the force matrix (I is None)."""
        n = self.n
        phi = np.zeros(n, np.int32)
        I = np.zeros((n, n), np.int64) if force else None
        E = np.zeros(1, np.int64)
        bE = np.zeros(1, np.int64)
        b = np.zeros(1, np.float64)
        _check(lib().pimqap_solver_replica(self.h, t, l, phi.ctypes.data, I.ctypes.data if force else None,
                                           E.ctypes.data, bE.ctypes.data, b.ctypes.data))
        return dict(phi=phi, I=I, E=int(E[0]), bestE=int(bE[0]), beta=float(b[0]))

    def events(self, first: int = 0) -> List[dict]:
        """Progress events recorded so far (params.event_capacity > 0), in the reference's order."""
        total = C.c_int64(0)
        dropped = C.c_int64(0)
        count = C.c_int32(0)
        _check(lib().pimqap_solver_events(self.h, 0, 0, None, C.byref(count), C.byref(total), C.byref(dropped)))
        k = max(0, total.value - first)
        buf = (Event * max(1, k))()
        _check(lib().pimqap_solver_events(self.h, first, k, buf, C.byref(count), None, None))
        self.events_dropped = dropped.value
        return [_event_dict(buf[i]) for i in range(count.value)]

    def event_perm(self, perm_index: int) -> np.ndarray:
        perm = np.zeros(self.n, np.int32)
        _check(lib().pimqap_solver_event_perm(self.h, perm_index, perm.ctypes.data))
        return perm

    def group(self, t: int, rank_slots: int) -> dict:
        order = np.zeros(rank_slots, np.int32)
        tss = np.zeros(1, np.int32)
        gb = np.zeros(1, np.int64)
        _check(lib().pimqap_solver_group(self.h, t, order.ctypes.data, tss.ctypes.data, gb.ctypes.data))
        return dict(order=order, time_since_swap=int(tss[0]), group_best=int(gb[0]))

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().pimqap_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Server:
    """Continuous-batching solve service: submit() requests at any time, wait() / poll() for
    their results.  sample: optional list of (F, D, Params) representative of the expected
    requests, from which the autotuner sizes the resident launches."""

    def __init__(self, device: int = 0, memory_budget: int = 0, slots_per_class: int = 0,
                 heartbeat_timeout: float = 0.0, sample=None):
        cfg = ServerConfig()
        cfg.device = device
        cfg.memory_budget_bytes = memory_budget
        cfg.slots_per_class = slots_per_class
        cfg.heartbeat_timeout_s = heartbeat_timeout
        keep = []
        if sample:
            insts = [_Inst(F, D) for F, D, _ in sample]
            keep.append(insts)
            arr = (Instance * len(insts))(*[i.c for i in insts])
            parr = (Params * len(sample))(*[p for _, _, p in sample])
            keep += [arr, parr]
            cfg.sample = C.cast(arr, C.POINTER(Instance))
            cfg.sample_params = C.cast(parr, C.POINTER(Params))
            cfg.sample_count = len(sample)
        h = C.c_void_p()
        _check(lib().pimqap_server_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self._shapes = {}

    def submit(self, F: np.ndarray, D: np.ndarray, params: Params) -> int:
        inst = _Inst(F, D)
        t = C.c_int64(0)
        _check(lib().pimqap_server_submit(self.h, C.byref(inst.c), C.byref(params), C.byref(t)))
        self._shapes[t.value] = (inst.F.shape[0], params.groups * params.replicas)
        return t.value

    def _fetch(self, ticket: int, timeout: float):
        n, reps = self._shapes[ticket]
        r, perm, energies = _new_result(n, reps)
        st = lib().pimqap_server_wait(self.h, ticket, timeout, C.byref(r))
        if st == 8:      # not ready
            return None
        del self._shapes[ticket]
        _check(st)
        return _result_dict(r, perm, energies)

    def poll(self, ticket: int):
        return self._fetch(ticket, 0.0)

    def wait(self, ticket: int, timeout: float = -1.0) -> dict:
        out = self._fetch(ticket, timeout)
        if out is None:
            raise PimqapError(8, "request not finished within the timeout")
        return out

    def stats(self) -> dict:
        s = ServerStats()
        _check(lib().pimqap_server_stats_get(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def stall_heartbeat(self, stall: bool) -> None:
        lib().pimqap_server_debug_stall_heartbeat(self.h, 1 if stall else 0)

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().pimqap_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
