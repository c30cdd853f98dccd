"""The `pimqap` CLI on the GPU against the reference CLI's golden outputs, and the progress
event API (pimqap_solver_events) against the oracle.

The golden fixtures (tests/golden/cli_golden.json) hold the stdout, log.txt and sweep<t>.txt of
the reference's own main() (CPU-PIM/CPU_PIM.cpp:478-685) fed the solver's Philox streams; they
are pinned to the oracle by tests/test_cli.py.  With one group the reference prints in a fixed
order and every line must match; with several groups its threads race on the shared best, so
the sweep files and the final best must match.
"""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import instances
from helpers import LN2_INV, oracle_cli_trace
from test_cli import CLI, ROOT, golden

pytestmark = pytest.mark.gpu

TIME = re.compile(r"(Time \(s\): )\S+")
ELAPSED = re.compile(r"^(Elapsed time: )\S+( seconds\.)$")
TOOK = re.compile(r"^(Selecting Beta Parameters took )\d+( seconds\.)$")


def normalise(text):
    out = []
    for line in text.splitlines():
        line = TIME.sub(r"\1*", line)
        line = ELAPSED.sub(r"\1*\2", line)
        line = TOOK.sub(r"\1*\2", line)
        out.append(line)
    return out


def run_ours(c, out):
    inst = os.path.join("tests", "golden", "cli", c["instance"])
    cp = subprocess.run([CLI, "--seed", str(c["seed"])] + c["flags"] + ["-o", out, inst],
                        capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert cp.returncode == 0, cp.stderr
    with open(os.path.join(out, "log.txt")) as f:
        log = f.read()
    sweeps = {}
    for name in sorted(os.listdir(out)):
        m = re.fullmatch(r"sweep(\d+)\.txt", name)
        if m:
            with open(os.path.join(out, name)) as f:
                pairs = [[int(a), int(c_)] for a, _ms, c_ in (l.split() for l in f)]
            if pairs:
                sweeps[m.group(1)] = pairs
    return normalise(cp.stdout), normalise(log), sweeps


@pytest.mark.parametrize("name", [c["name"] for c in golden()["cases"]])
def test_cli_matches_reference_cli(gpu, name):
    c = next(c for c in golden()["cases"] if c["name"] == name)
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "out")
        stdout, log, sweeps = run_ours(c, out)
    assert sweeps == c["sweeps"]
    final = [l for l in c["stdout"] if l.startswith("Single best energy found")]
    assert [l for l in stdout if l.startswith("Single best energy found")] == final
    if c["ordered"]:
        assert stdout == c["stdout"]
        assert log == c["log"]
    else:
        assert log[:4] == c["log"][:4]


def test_solver_events_follow_the_oracle(gpu, oracle):
    inst = instances.uniform(28, 9001)
    T, R, spe, W = 3, 5, 2, 40
    b = 0.0003
    p = gpu.default_params(replicas=R, groups=T, sweeps_per_exchange=spe, beta_max=b, beta_ratio=1.25,
                           seed=17, max_megaiters=W, event_capacity=4096, megaiters_per_launch=7)
    with gpu.Solver(inst.F, inst.D, p) as s:
        s.run(W)
        ev = s.events()
    lines, sweeps, single = oracle_cli_trace(oracle, inst.F, inst.D, T=T, R=R, spe=spe, beta0=b * LN2_INV,
                                             ratio=1.25, seed=17, megaiters=W)
    got = [e for e in ev if e["kind"] == gpu.EVENT_GROUP_BEST and e["megaiter"] < W]
    # per group: the last event of each mega-iteration is the sweep<t>.txt pair
    for t in range(T):
        pairs = {}
        for e in got:
            if e["group"] == t:
                pairs[e["megaiter"]] = e["energy"]
        assert [[m, v] for m, v in sorted(pairs.items())] == sweeps[t]
    assert all(a["time_ms"] <= b_["time_ms"] + 1e-9 for a, b_ in zip(got, got[1:])
               if a["megaiter"] < b_["megaiter"])
    single_ev = min(e["energy"] for e in got)
    assert single_ev == single


def test_goal_print_events_carry_their_permutation(gpu, oracle):
    inst = instances.uniform(24, 77)
    p = gpu.default_params(replicas=4, groups=2, sweeps_per_exchange=2, beta_max=0.0002, beta_ratio=1.3,
                           seed=9, max_megaiters=60, event_capacity=4096, goal_print=1110000)
    with gpu.Solver(inst.F, inst.D, p) as s:
        s.run(60)
        ev = [e for e in s.events() if e["kind"] == gpu.EVENT_GOAL_PRINT]
        assert ev, "no replica went below goal_print"
        F = inst.F.astype(np.int64)
        D = inst.D.astype(np.int64)
        for e in ev:
            assert e["energy"] < 1110000 and e["perm_index"] >= 0
            phi = s.event_perm(e["perm_index"])
            assert sorted(phi.tolist()) == list(range(24))
            assert int((D * F[np.ix_(phi, phi)]).sum()) == e["energy"]
        # each replica's goal-print energies strictly decrease, in mega-iteration order
        for t in range(2):
            for l in range(4):
                es = [e for e in ev if e["group"] == t and e["replica"] == l]
                assert all(a["megaiter"] <= b["megaiter"] and a["energy"] > b["energy"] for a, b in zip(es, es[1:]))
