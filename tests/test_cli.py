"""The `pimqap` CLI as a drop-in for the reference's CPU_PIM binary (CPU-PIM/CPU_PIM.cpp:478-685).

CPU only: the golden outputs of the reference CLI (tests/golden/cli_golden.json, recorded by
tests/golden/make_cli_golden.py from the reference's own main() fed the solver's Philox
streams) are pinned to the oracle, and the CLI's argument and file errors are checked (they
come before any GPU work).  The GPU side of the comparison is tests/test_gpu_cli.py.
"""
import json
import os
import re
import subprocess

import pytest

import instances
from helpers import LN2_INV, oracle_auto_beta, oracle_cli_trace, splitmix64, MASK64
from oracle import REF_DIR

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "cli_golden.json")
CLI = os.path.join(ROOT, "p-dit-probabilistic-ising-machine-for-solving-the-quadratic-assignment-problem_b200",
                   "csrc", "pimqap")


def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def case(name):
    return next(c for c in golden()["cases"] if c["name"] == name)


def flag(c, name, cast=float, default=None):
    f = c["flags"]
    return cast(f[f.index(name) + 1]) if name in f else default


def best_found(lines):
    return [int(l.split()[3]) for l in lines if l.startswith("Best Energy Found:")]


def load(c):
    inst = instances.read_instance(os.path.join(ROOT, "tests", "golden", "cli", c["instance"]))
    return inst.F, inst.D


@pytest.mark.parametrize("name", ["fixed_t1", "fixed_t3", "fixed_t2_i1", "goal_t1"])
def test_golden_fixed_beta_runs_match_oracle(oracle, name):
    c = case(name)
    F, D = load(c)
    T, R = flag(c, "-t", int), flag(c, "-r", int)
    lines, sweeps, single = oracle_cli_trace(
        oracle, F, D, T=T, R=R, spe=flag(c, "-i", int), beta0=flag(c, "-b") * LN2_INV,
        ratio=flag(c, "-m"), seed=c["seed"], megaiters=flag(c, "-w", int), goal=flag(c, "-g", int, 0))
    assert {str(t): s for t, s in sweeps.items() if s} == c["sweeps"]
    assert f"Single best energy found: {single}" in c["stdout"]
    if c["ordered"]:
        assert best_found(c["stdout"]) == lines


def test_golden_automatic_mode_matches_oracle(oracle):
    c = case("auto_t1")
    F, D = load(c)
    T, R, spe, W, seed = flag(c, "-t", int), flag(c, "-r", int), flag(c, "-i", int), flag(c, "-w", int), c["seed"]
    b0, db, sums, _ = oracle_auto_beta(oracle, F, D, T=T, R=R, spe=spe, seed=seed, cap=10)
    beta_lines = [l for l in c["stdout"] if l.startswith("Beta: ")]
    assert beta_lines == [f"Beta: {2.0 ** (-30 + i):g}, Average Energy: {sums[i]:g}" for i in range(32)]
    assert f"Maximum Beta {b0:g}" in c["stdout"]
    assert f"Multiplicative Beta between iterations {db:g}" in c["stdout"]
    # "Best Energy Found" lines: the 160 trials in order, then the run, sharing the best
    single, expect = 2147483647, []
    for k in range(160):
        lines, _, single = oracle_cli_trace(oracle, F, D, T=T, R=R, spe=spe, beta0=2.0 ** (-30 + k // 5),
                                            ratio=1.0, seed=splitmix64((seed + k + 1) & MASK64),
                                            megaiters=10, single=single)
        expect += lines
    lines, sweeps, single = oracle_cli_trace(oracle, F, D, T=T, R=R, spe=spe, beta0=b0, ratio=db, seed=seed,
                                             megaiters=W, single=single)
    expect += lines
    assert best_found(c["stdout"]) == expect
    assert c["sweeps"] == {str(t): s for t, s in sweeps.items() if s}
    assert f"Single best energy found: {single}" in c["stdout"]


def test_golden_reproduced_by_reference_cli():
    """The committed fixtures are what the reference CLI prints (where it is built)."""
    if not os.path.exists(os.path.join(REF_DIR, "cpu_pim_philox")):
        pytest.skip("reference CLI not built here (oracle/_ref)")
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_cli_golden", os.path.join(ROOT, "tests", "golden",
                                                                                  "make_cli_golden.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    cwd = os.getcwd()
    os.chdir(ROOT)
    try:
        import tempfile
        for c in golden()["cases"]:
            with tempfile.TemporaryDirectory() as d:
                so, log, sweeps = mk.run_ref(os.path.join("tests", "golden", "cli", c["instance"]), c["seed"],
                                             c["flags"], d)
            assert sweeps == c["sweeps"], c["name"]
            if c["ordered"]:
                assert mk.normalise(so) == c["stdout"], c["name"]
                assert mk.normalise(log) == c["log"], c["name"]
    finally:
        os.chdir(cwd)


def run_cli(args, cwd):
    if not os.path.exists(CLI):
        pytest.fail(f"{CLI} is not built (make -C csrc)")
    return subprocess.run([CLI] + args, capture_output=True, text=True, cwd=cwd, timeout=60)


def test_help_is_the_reference_usage():
    out = run_cli(["--help"], ROOT).stdout.splitlines()
    ref = golden()["help"]
    assert out[1:1 + len(ref)] == ref
    assert out[0].startswith("Usage: ") and out[0].endswith(" [OPTIONS]... [FILE]...")


def test_argument_and_file_errors(tmp_path):
    r = run_cli([], str(tmp_path))
    assert r.returncode == 1 and "Error: No input file specified." in r.stderr
    r = run_cli(["-o", "outdir", "missing.dat"], str(tmp_path))
    assert r.returncode == 1 and "Error: Could not open the file (missing.dat)." in r.stderr
    assert (tmp_path / "outdir").is_dir()          # the folder comes first (:617-631)
    big = tmp_path / "big.dat"
    big.write_text("300\n")
    r = run_cli([str(big)], str(tmp_path))
    assert r.returncode == 1 and "Error: N exceeded MAXN (256)." in r.stderr
    assert (tmp_path / "big.dat.out").is_dir()      # default folder name (:613-615)
    r = run_cli(["-r", "65", str(big)], str(tmp_path))
    assert r.returncode == 1 and "exceeds maximum number of replicas (64)" in r.stderr
    r = run_cli(["-w"], str(tmp_path))
    assert r.returncode == 1 and "Error: -w option requires a value." in r.stderr
    r = run_cli(["-g", "abc", str(big)], str(tmp_path))
    assert r.returncode == 1 and "numeric" in r.stderr
