"""The C ABI library loads, exports every declared entry point, and validates arguments and
files without touching a GPU (CPU only)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import instances
import pimqap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pimqap.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^[A-Za-z_][\w ]*?\**\s*\**(pimqap_\w+)\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert "pimqap_solve" in names and "pimqap_read_problem" in names
    out = subprocess.run(["nm", "-D", "--defined-only", pimqap.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (pimqap_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    L = pimqap.lib()
    for n in names:
        assert hasattr(L, n)


def test_default_params_mirror_reference_defaults():
    p = pimqap.default_params()
    assert (p.replicas, p.groups, p.sweeps_per_exchange) == (10, 20, 4)
    assert p.beta_ratio == 1.2 and p.goal == 0
    assert abs(p.beta_max * pimqap.LN2_INV - 2.0 ** -12) < 1e-15


def test_read_problem_round_trip(tmp_path):
    inst = instances.heavy(41, 3)
    path = str(tmp_path / "h41.dat")
    instances.write_instance(path, inst)
    F, D = pimqap.read_problem(path)
    assert np.array_equal(F, inst.F) and np.array_equal(D, inst.D)


def test_load_file_allocates_and_frees(tmp_path):
    inst = instances.uniform(29, 4)
    path = str(tmp_path / "u29.dat")
    instances.write_instance(path, inst)
    F, D = pimqap.load_file(path)
    assert np.array_equal(F, inst.F) and np.array_equal(D, inst.D)
    with pytest.raises(pimqap.PimqapError) as e:
        pimqap.load_file(str(tmp_path / "missing.dat"))
    assert e.value.status == 2
    empty = pimqap.Instance()
    pimqap.lib().pimqap_free_instance(C.byref(empty))     # freeing an empty instance is a no-op
    assert empty.n == 0


def test_replay_and_batch_arguments_are_checked():
    inst = instances.uniform(6, 1)
    p = pimqap.default_params(replicas=1, groups=1, beta_max=0.1)
    with pytest.raises(pimqap.PimqapError) as e:             # not a permutation
        pimqap.sweep_replay(inst.F, inst.D, p, np.array([0, 0, 1, 2, 3, 4]), np.full((1, 6), 0.5))
    assert e.value.status == 1
    with pytest.raises(pimqap.PimqapError) as e:             # r outside [0, 1)
        pimqap.sweep_replay(inst.F, inst.D, p, np.arange(6), np.full((1, 6), 1.0))
    assert e.value.status == 1
    p.update_rule = pimqap.RULE_ONE_SHOT
    with pytest.raises(pimqap.PimqapError):
        pimqap.sweep_replay(inst.F, inst.D, p, np.arange(6), np.full((1, 6), 0.5))
    h = C.c_void_p()
    assert pimqap.lib().pimqap_batch_submit(None, None, 0, None, C.byref(h)) == 1
    assert pimqap.lib().pimqap_batch_poll(None) == 1


def test_read_problem_errors(tmp_path):
    with pytest.raises(pimqap.PimqapError) as e:
        pimqap.read_problem(str(tmp_path / "missing.dat"))
    assert e.value.status == 2
    big = instances.uniform(30, 1)
    path = str(tmp_path / "u30.dat")
    instances.write_instance(path, big)
    with pytest.raises(pimqap.PimqapError) as e:      # the reference's MAXN check
        pimqap.read_problem(path, max_n=20)
    assert e.value.status == 1 and "MAXN" in str(e.value)
    trunc = tmp_path / "trunc.dat"
    trunc.write_text("3\n1 2 3\n4 5 6\n")
    with pytest.raises(pimqap.PimqapError) as e:
        pimqap.read_problem(str(trunc))
    assert e.value.status == 2


# Both solve entry points take the same parameters and reject the same invalid ones before
# touching a device: the solver handle (pimqap_solver_create, behind pimqap_solve) and the
# allocation-free pimqap_solve_static.
ENTRY_POINTS = {
    "solver": lambda inst, p: pimqap.Solver(inst.F, inst.D, p),
    "solve_static": lambda inst, p: pimqap.solve_static(inst.F, inst.D, p),
}


@pytest.mark.parametrize("entry", sorted(ENTRY_POINTS))
@pytest.mark.parametrize("field,value", [("replicas", 0), ("replicas", 65), ("groups", 0),
                                         ("sweeps_per_exchange", 0), ("beta_max", 0.0),
                                         ("beta_ratio", -1.0), ("force_bits", 16),
                                         ("threads_per_block", 96), ("rank_slots", 2),
                                         ("timeout_s", -1.0), ("timeout_s", float("nan")),
                                         ("timeout_s", float("inf"))])
def test_invalid_params_rejected_before_device(entry, field, value):
    inst = instances.uniform(8, 1)
    p = pimqap.default_params(replicas=4, groups=1, max_megaiters=1)
    setattr(p, field, value)
    with pytest.raises(pimqap.PimqapError) as e:
        ENTRY_POINTS[entry](inst, p)
    assert e.value.status == 1


@pytest.mark.parametrize("entry", sorted(ENTRY_POINTS))
@pytest.mark.parametrize("fields", [{"update_rule": 2}, {"cluster_size": 3}, {"compact_instance": 2},
                                    {"active_facilities": 1}, {"active_facilities": -3},
                                    {"active_facilities": 8},
                                    {"max_megaiters": -1}, {"event_capacity": -1},
                                    {"threads_per_block": 512},
                                    {"update_rule": 1, "active_facilities": 4},
                                    {"replica_pairing": 3}, {"replica_pairing": -1},
                                    {"launch_mode": 3}, {"launch_mode": -1},
                                    {"threads_per_block": 32, "update_rule": 1},
                                    {"sweep_pipeline": 3}, {"sweep_pipeline": -1},
                                    {"tensor_update": 4}, {"tensor_update": -1},
                                    {"tensor_update": 2},
                                    {"oneshot_weights": 2}, {"oneshot_weights": -1}])
def test_invalid_combinations_rejected_before_device(entry, fields):
    inst = instances.uniform(8, 1)
    p = pimqap.default_params(replicas=4, groups=1, max_megaiters=1)
    for k, v in fields.items():
        setattr(p, k, v)
    with pytest.raises(pimqap.PimqapError) as e:
        ENTRY_POINTS[entry](inst, p)
    assert e.value.status == 1
    if fields == {"update_rule": 2}:
        assert "update_rule must be" in str(e.value)


@pytest.mark.parametrize("fields,msg", [({"auto_beta": 1}, "automatic beta"),
                                        ({"active_facilities": 4}, "active_facilities"),
                                        ({"update_rule": 1}, "one-shot")])
def test_static_solve_rejects_what_it_does_not_run(fields, msg):
    """Valid for pimqap_solve, but not run by the allocation-free entry point."""
    inst = instances.uniform(8, 1)
    p = pimqap.default_params(replicas=4, groups=1, max_megaiters=1)
    for k, v in fields.items():
        setattr(p, k, v)
    with pytest.raises(pimqap.PimqapError) as e:
        pimqap.solve_static(inst.F, inst.D, p)
    assert e.value.status == 1 and msg in str(e.value) and "pimqap_solve" in str(e.value)


def test_valid_solve_without_a_gpu_fails_loudly():
    """No CPU fallback: with no sm_100 device a valid solve reports PIMQAP_ERR_NO_DEVICE."""
    from conftest import _has_gpu
    if _has_gpu():
        pytest.skip("a GPU is visible")
    inst = instances.uniform(8, 1)
    with pytest.raises(pimqap.PimqapError) as e:
        pimqap.solve(inst.F, inst.D, pimqap.default_params(replicas=2, groups=1, max_megaiters=1))
    assert e.value.status == 4


def test_n_out_of_range_rejected():
    F = np.zeros((257, 257), np.int32)
    with pytest.raises(pimqap.PimqapError) as e:
        pimqap.Solver(F, F, pimqap.default_params())
    assert e.value.status == 1


def test_release_kept_memory_with_nothing_kept_makes_no_cuda_call():
    # no solve has run in this process, so nothing is kept and no GPU is needed
    pimqap.release_kept_memory()
