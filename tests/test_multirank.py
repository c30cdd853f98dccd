"""The multi-GPU layout of bench.py, on CPU: two `gloo` ranks (world_size 2).

One process per GPU; each rank solves its own instance (sharding by instance, no data-path
collective); the timed figure is the slowest rank's time, and the whole-job rate counts every
rank's work.  The reference arm runs on rank 0 only.
"""
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        inst = bench.rank_instance(rank)
        ms = 10.0 * (rank + 1)                      # rank 1 is the slower one
        ms_max = bench.max_over_ranks(ms, world, "cpu")
        rate = bench.whole_job_rate(1000.0, world, ms_max * 1e-3)
        out.put((rank, int(inst.F.sum()), ms_max, rate))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_instances_and_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, f0, m0, v0), (r1, f1, m1, v1) = got
    assert f0 != f1                                   # different instances per rank
    assert m0 == m1 == 20.0                           # max over ranks, the same on every rank
    assert v0 == v1 == 1000.0 * 2 / 0.020             # all ranks' units / slowest time


def test_reference_arm_prints_only_on_rank_zero():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "3", "--warmup", "3"], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_names_the_solver_arms_workload():
    """Rank 0 times the reference's CPU program on the workload the solver's arm names (the same
    config keys but the parallelism), and reports what it cannot time instead of timing
    something else."""
    import json
    sys.path.insert(0, ROOT)
    import bench
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--update-rule", "one-shot", "--steps", "3", "--warmup", "3"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "3"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0
    line = json.loads(r.stdout.strip().splitlines()[-1])
    if "unavailable" in line:                         # oracle/_ref not built here
        return
    want = bench.workload_config("grid256", "sequential", 1, 1)
    got = dict(line["config"])
    assert got.pop("parallelism") != want.pop("parallelism")
    assert got == want
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT and line["higher_is_better"]
    assert line["e2e"]["value"] == line["value"] == line["cpu_baseline"]["value"] > 0
