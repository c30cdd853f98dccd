#!/usr/bin/env python
"""Benchmark of the B200 p-dit QAP solver: swap proposals per second.

Workload (one instance per GPU, weak scaling over GPUs): n = 256, flow a symmetric
Bernoulli(0.36) 0/1 matrix, distance the squared Euclidean distance on a 16 x 16 integer grid
plus a symmetric uniform [0, 3] perturbation (seeded synthetic stand-in for the published
single-instance workload), 64 replicas on one geometric beta ladder, replica exchange every
4 sweeps (the reference's NUMITERA default), 10^4 sweeps = 100 steps of 100 sweeps.

A "step" is 25 mega-iterations = 100 sweeps of all 64 replicas.  Proposals are counted as
the published metric defines them: n (n - 1) / 2 per sweep per replica.  --workload cfg1 runs
the reference's CPU-sized case instead (n = 32, 16 replicas, exchange every sweep; a step is
100 sweeps, so --steps 10 is its 1000 sweeps); --workload clique92 the tai256c structure.

  value       device-timed throughput with the instance resident in HBM (CUDA events on
              the solver's stream, L2 flushed between steps, max over ranks)
  e2e         the same work through the C ABI (pimqap_solve) from pinned host buffers:
              upload, set-up, all sweeps and the read-back of the result, host wall clock
  roofline    the sweep kernel against shared-memory read-modify-write bandwidth measured on
              this GPU (the force matrices are resident in shared memory), plus its HBM traffic
  cpu_baseline  the reference's own CPU_PIM.cpp (built from its source, oracle/_ref) on the
              host cores, one parallel-tempering group per thread

--impl reference times the reference's CPU implementation alone (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "p-dit-probabilistic-ising-machine-for-solving-the-quadratic-assignment-problem_b200")
sys.path.insert(0, PKG)

import instances  # noqa: E402

N = 256
REPLICAS = 64
SWEEPS_PER_EXCHANGE = 4
MEGAITERS_PER_STEP = 25
# Geometric ladder chosen by the reference's automatic mode (pimqap_auto_beta on this
# instance, 64 replicas, seed 1: beta0 = 2^-5 in the reference's internal log2 units, deltaBeta
# = 64^(1/64)), then fixed for the run.
BETA_MAX = 2.0 ** -5           # internal units
BETA_RATIO = 1.0671404006768237
# Ladders of the batch / serving suites, chosen the same way on representative instances.
LADDER_UNIFORM = (2.0 ** -9, 1.1387886347566916)    # uniform n = 85, 32 replicas
LADDER_HEAVY = (2.0 ** -13, 1.0787607977571199)     # heavy-tailed n = 180, 64 replicas
METRIC = "swap proposals/sec"
UNIT = "proposals/s"
L2_FLUSH_BYTES = 256 << 20
E2E_SOLVES = 3                  # end-to-end solves timed; the median wall is reported


# Workloads of the headline line.  grid256 is the driver's default (the published single-GPU
# configuration); clique92 is the structure the reference's tai256c program is written for;
# cfg1 is the reference's own CPU-sized case (n = 32, 16 replicas, beta 0.01 .. 10 natural,
# exchange every sweep, 1000 sweeps).
WORKLOADS = {
    "grid256": dict(n=N, replicas=REPLICAS, spe=SWEEPS_PER_EXCHANGE, megaiters_per_step=MEGAITERS_PER_STEP,
                    beta0=BETA_MAX, ratio=BETA_RATIO, act=0,
                    instance=lambda rank: instances.grid256(1000 + rank),
                    ladder="reference automatic mode on this instance (pimqap_auto_beta, seed 1), then fixed",
                    desc="grid256: n=256 Bernoulli(0.36) flow, 16x16 grid sq. distance + U[0,3]; 64 replicas, "
                         "geometric beta ladder, exchange every 4 sweeps"),
    "clique92": dict(n=N, replicas=REPLICAS, spe=SWEEPS_PER_EXCHANGE, megaiters_per_step=MEGAITERS_PER_STEP,
                     beta0=BETA_MAX, ratio=BETA_RATIO, act=92,
                     instance=lambda rank: instances.clique_flow(1000 + rank),
                     ladder="the grid256 ladder",
                     desc="clique92: n=256, unit flows among facilities 0..91, 16x16 grid sq. distance + U[0,3]; "
                          "the tai256c program's moves; 64 replicas, geometric beta ladder, exchange every 4 sweeps"),
    "cfg1": dict(n=32, replicas=16, spe=1, megaiters_per_step=100,
                 beta0=10.0 * 1.44269504089, ratio=1.5849, act=0,
                 instance=lambda rank: instances.uniform(32, 1000 + rank),
                 ladder="geometric 0.01 .. 10 in natural units (-b 10 -m 1.5849)",
                 desc="cfg1: n=32, symmetric uniform [0,99] flow and distance, zero diagonal; 16 replicas, "
                      "beta 0.01 .. 10 natural, exchange every sweep; the published 1000 sweeps are --steps 10"),
}


def proposals(replicas: int, sweeps: int, n: int = N) -> float:
    return float(replicas) * sweeps * n * (n - 1) / 2.0


# ------------------------------------------------------------------ clocks

REASON_BITS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
               0x8: "hw_slowdown", 0x10: "sync_boost", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
               0x100: "display_clock_setting"}


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        cmd = ["nvidia-smi", "-i", str(self.device),
               "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active",
               "--format=csv,noheader,nounits", "-lms", "200"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 4:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
                bits = int(parts[3], 16)
            except ValueError:
                continue
            for b, name in REASON_BITS.items():
                if bits & b and name != "gpu_idle":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ reference CPU timing

def ref_cpu_throughput(F, D, budget_s: float, W: dict):
    """The reference's threadToRun on one thread per host core for ~budget_s seconds.
    Returns (proposals/s, cores, kind, sample description) or None."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import RefHarness, ref_available
    if not ref_available("big_mt"):
        return None
    ref = RefHarness("big_mt")
    cores = max(1, min(os.cpu_count() or 1, ref.maxt))
    ref.load(F, D)
    ref.setup_replicated(cores, W["replicas"], W["spe"], W["beta0"], W["ratio"], 1)
    t1 = ref.run(1)
    m = max(1, int(budget_s / max(t1, 1e-3)))
    el = ref.run(m)
    sweeps = m * W["spe"]
    val = proposals(cores * W["replicas"], sweeps, W["n"]) / el
    sample = (f"{cores} threads x {W['replicas']} replicas of the n={W['n']} instance, {sweeps} sweeps each "
              f"({m} mega-iterations of {W['spe']} sweeps), {el:.1f} s")
    return val, cores, "reference", sample


def workload_config(workload, update_rule, world, steps, groups=1):
    """The workload part of the line's config, the same in both arms; it names the sweeps the
    timed region actually runs.  groups > 1: that many independent parallel-tempering groups of
    the workload's replicas (the reference's -t threads) on each GPU."""
    W = WORKLOADS[workload]
    sweeps = steps * W["megaiters_per_step"] * W["spe"]
    return {"workload": W["desc"] + f"; {sweeps} sweeps timed ({steps} steps of "
                                     f"{W['megaiters_per_step'] * W['spe']})" +
                        ("; GPU-CUPIM's one-shot rule (a sweep = one parallel step)"
                         if update_rule == "one-shot" else ""),
            "update_rule": update_rule,
            "n": W["n"], "replicas": W["replicas"] * groups, "groups": groups,
            "sweeps_per_step": W["megaiters_per_step"] * W["spe"], "sweeps_per_exchange": W["spe"],
            "beta0_internal": W["beta0"], "beta_ratio": W["ratio"],
            "ladder": W["ladder"],
            "sweeps_timed": sweeps,
            "parallelism": f"instances x{world}"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import RefHarness, ref_available
    if args.workload == "clique92" or args.update_rule != "sequential":
        print(json.dumps({"impl": "reference", "unavailable": "the reference arm times the grid256 and cfg1 "
                                                              "workloads with the sequential rule (CPU_PIM.cpp) only"}))
        return
    W = WORKLOADS[args.workload]
    cfg = dict(workload_config(args.workload, args.update_rule, 1, args.steps, args.groups),
               parallelism="host threads (the reference's CPU program; no GPU)")
    if not ref_available("big_mt"):
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU_PIM.cpp not built (oracle/_ref missing)"}))
        return
    inst = W["instance"](0)
    ref = RefHarness("big_mt")
    cores = max(1, min(os.cpu_count() or 1, ref.maxt))
    ref.load(inst.F, inst.D)
    ref.setup_replicated(cores, W["replicas"], W["spe"], W["beta0"], W["ratio"], 1)
    t1 = ref.run(1)
    # each step a bounded sample: the whole run stays within ~3 minutes
    per_step = min(2.0, 180.0 / max(1, args.steps + args.warmup))
    m = max(1, int(per_step / max(t1, 1e-3)))
    for _ in range(args.warmup):
        ref.run(m)
    total = 0.0
    for _ in range(args.steps):
        total += ref.run(m)
    sweeps = args.steps * m * W["spe"]
    val = proposals(cores * W["replicas"], sweeps, W["n"]) / total
    sample = (f"each step {m} mega-iterations ({W['spe']} sweeps each) of {cores} groups x {W['replicas']} "
              f"replicas of the n={W['n']} instance; one group per host thread")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": f"synthetic (seeded {args.workload} instance)", "config": cfg,
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference's CPU program on this host's cores; no GPU is used at any n_gpus"}
    print(json.dumps(line))


# ------------------------------------------------------------------ our arm

def rank_instance(rank, workload="grid256"):
    """The instance rank `rank` solves: one instance per GPU (the work is sharded by
    instance; ranks never exchange data)."""
    return WORKLOADS[workload]["instance"](rank)


def max_over_ranks(x, world, device):
    """The largest x over all ranks (the slowest rank bounds the whole job)."""
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, world, seconds_max):
    """Units all ranks processed / the slowest rank's time."""
    return units_per_rank * world / seconds_max


def run_ours(args):
    import torch
    import torch.distributed as dist
    import pimqap

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus and "WORLD_SIZE" in os.environ:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    W = WORKLOADS[args.workload]
    n, reps, spe, MPS = W["n"], W["replicas"] * args.groups, W["spe"], W["megaiters_per_step"]
    inst = rank_instance(rank, args.workload)
    rule = pimqap.RULE_ONE_SHOT if args.update_rule == "one-shot" else pimqap.RULE_SEQUENTIAL
    common = dict(replicas=W["replicas"], groups=args.groups, sweeps_per_exchange=spe, beta_max=W["beta0"],
                  beta_ratio=W["ratio"], beta_internal=1, seed=1 + rank, device=local,
                  cluster_size=args.cluster_size, threads_per_block=args.threads,
                  active_facilities=W["act"], update_rule=rule, replica_pairing=args.pairing,
                  launch_mode=args.launch_mode, sweep_pipeline=args.pipeline,
                  tensor_update=args.tensor_update)
    params = pimqap.default_params(megaiters_per_launch=MPS, max_megaiters=2 ** 31 - 1, **common)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{local}")
    solver = pimqap.Solver(inst.F, inst.D, params)
    for _ in range(args.warmup):
        solver.run(MPS)
    r0 = solver.result()

    def barrier():
        if world > 1:
            dist.barrier()

    # e2e first: the same work through the C ABI (pimqap_solve) from pinned host buffers,
    # before the clock sampler's process runs
    Fp = torch.from_numpy(inst.F).pin_memory()
    Dp = torch.from_numpy(inst.D).pin_memory()
    p2 = pimqap.default_params(megaiters_per_launch=4 * MPS,   # fewer host round trips
                               max_megaiters=args.steps * MPS, **common)
    # one untimed call of the same API (one mega-iteration) takes any first-call cost of the
    # process (module loading, first graph of this shape) out of the timed call
    pw = pimqap.Params.from_buffer_copy(p2)
    pw.max_megaiters = 1
    pimqap.solve(Fp.numpy(), Dp.numpy(), pw)
    # three timed solves, the median wall reported (a single solve of under a second saw the
    # host's scheduling noise: 0.70 to 1.48 s for the same device time)
    e_runs = []
    for _ in range(E2E_SOLVES):
        barrier()
        e0 = time.perf_counter()
        res = pimqap.solve(Fp.numpy(), Dp.numpy(), p2)
        e_runs.append((time.perf_counter() - e0, res))
    e_walls = [w for w, _ in e_runs]
    e_wall, res = sorted(e_runs, key=lambda x: x[0])[len(e_runs) // 2]
    e2e_sweeps = args.steps * MPS * spe
    e2e_value = whole_job_rate(proposals(reps, e2e_sweeps, n), world,
                               max_over_ranks(e_wall, world, f"cuda:{local}"))

    ms_total = 0.0
    with ClockSampler(local) as clocks:
        barrier()
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            ms_total += solver.run(MPS)
        torch.cuda.synchronize()
        barrier()
        wall = time.perf_counter() - w0
    r1 = solver.result()
    solver.close()
    ms_max = max_over_ranks(ms_total, world, f"cuda:{local}")
    sweeps = args.steps * MPS * spe
    value = whole_job_rate(proposals(reps, sweeps, n), world, ms_max * 1e-3)

    # roofline of the sweep kernel (every timed launch is that kernel)
    accepts = r1["accepts"] - r0["accepts"]
    cand = float(reps) * sweeps * n * n
    s = r1["force_bits"] // 8
    if rule == pimqap.RULE_ONE_SHOT:
        # one read-modify-write of the force matrix per replica step, whatever the number of
        # swaps it applies, plus the swaps' D / F rows
        alg_bytes = (3 * s + 20) * cand + 2 * n * n * s * float(reps) * sweeps + 32 * n * float(accepts)
        bytes_model = f"({3 * s}+20) B per candidate delta + 2 n^2 {s} B per replica step + 32 n B per accept"
    else:
        alg_bytes = (3 * s + 20) * cand + (2 * n * n * s + 32 * n) * float(accepts)
        bytes_model = f"({3 * s}+20) B per candidate delta + (2 n^2 {s} + 32 n) B per accept"
    launches = r1["launches"] - r0["launches"]
    persistent = launches == args.steps
    achieved = alg_bytes / (ms_total * 1e-3) / 1e9
    smem_peak = pimqap.probe_smem_bandwidth(local)
    # HBM bytes every mega-iteration moves by construction: each replica's state is loaded into
    # shared memory and stored back (force rows, permutation, best permutation; the scalars are
    # noise), and every CTA stages the instance (D and F rows read as int32).  Measured DRAM bytes
    # come from ncu captures, not from this run.
    cl = r1["cluster_size"]
    npad = (n + 3) & ~3
    state_bytes = reps * (2 * n * npad * s + 3 * n * 4)
    stage_bytes = reps * cl * 2 * n * npad * 4

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline and args.workload != "clique92" and rule == 0:
            got = ref_cpu_throughput(inst.F, inst.D, 12.0, W)
            if got:
                v, cores, kind, sample = got
                cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": f"int{8 * s}",
            "data": f"synthetic (seeded {args.workload} instance per GPU)",
            "config": dict(workload_config(args.workload, args.update_rule, world, args.steps, args.groups),
                           cluster_size=r1["cluster_size"], force_bits=r1["force_bits"],
                           replica_pairing=args.pairing, sweep_pipeline=args.pipeline,
                           tensor_update=args.tensor_update,
                           launch="one persistent launch per step" if persistent else
                                  "a CUDA graph of one launch per mega-iteration",
                           l2="flushed between steps (256 MiB write)"),
            "candidate_deltas_per_s": cand * world / (ms_max * 1e-3),
            "accept_rate": accepts / (reps * sweeps * n),
            "best_energy": r1["best_energy"],
            "gpu_launches": launches,
            "wall_s_timed_region": wall,
            "roofline": {"bound": "smem", "achieved": achieved, "peak": smem_peak, "unit": "GB/s",
                         "frac": achieved / smem_peak,
                         "peak_source": "measured on this GPU by pimqap_probe_smem_bandwidth (shared-memory "
                                        "read-modify-write, 128-bit, 2 CTAs/SM)",
                         "traffic": None,
                         "traffic_note": "not measured in this run (no profiler in the timed region); "
                                         "ncu DRAM bytes per launch are in the committed profile summary",
                         "hbm_bytes_per_megaiter_by_construction": state_bytes + stage_bytes,
                         "alg_bytes_per_launch": alg_bytes / max(1, launches),
                         "bytes_model": bytes_model},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": res["h2d_bytes"],
                    "d2h_bytes_per_step": res["d2h_bytes"], "wall_s": e_wall,
                    "wall_s_each": e_walls, "library_wall_ms": res["wall_ms"], "device_ms": res["device_ms"],
                    "library_wall_ms_each": [r["wall_ms"] for _, r in e_runs],
                    "device_ms_each": [r["device_ms"] for _, r in e_runs],
                    "note": f"one step = one pimqap_solve of the whole workload (upload, set-up, sweeps, "
                            f"result); median wall of {E2E_SOLVES} solves"},
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return line


# ------------------------------------------------------------------ batch and serving suites

def _sweeps_proposals(n: int, replicas: int, sweeps: int) -> float:
    return float(replicas) * sweeps * n * (n - 1) / 2.0


def _ref_best(F, D, replicas, sweeps, b0, ratio, seconds_cap=120.0):
    """Best energy the reference's own CPU code (oracle/_ref, its std::mt19937 seeded from
    random_device) reaches on one instance: one parallel-tempering group per host thread, each
    `sweeps` sweeps (fewer when that would pass seconds_cap).  None when it is not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import RefHarness, ref_available
    if not ref_available("big_mt"):
        return None
    ref = RefHarness("big_mt")
    cores = max(1, min(os.cpu_count() or 1, ref.maxt))
    ref.load(F, D)
    ref.setup_replicated(cores, replicas, 4, b0, ratio, 1)
    t1 = ref.run(1)
    m = max(1, min(sweeps // 4, int(seconds_cap / max(t1, 1e-4))))
    el = ref.run(m - 1) if m > 1 else 0.0
    best = min(min(ref.replica(t, l)["bestE"] for l in range(replicas)) for t in range(cores))
    best = min(best, ref.single_best())
    return {"best": int(best), "groups": cores, "sweeps": 4 * m, "seconds": t1 + el}


def run_ttt_suite(args, name, batch, replicas, ladder, budget, plain_every, xcheck):
    """One batch of `batch` instances, `replicas` replicas each on `ladder`, `budget` sweeps:

    - the autotuner's choice per class (pimqap_batch_tune) and the fixed-work batch with the
      tuned shapes and with the fixed rules' shapes (PIMQAP_AUTOTUNE=0): proposals/s of each;
    - targets: the best energy of a run four times as long (other seeds), cross-checked on
      `xcheck` instances against the reference's own CPU code (best over one group per host
      thread) - a target above the reference's best is reported;
    - time to target (gap <= 0.1 %) of the batch and of the plain form (one pimqap_solve per
      instance, one instance per launch, every `plain_every`-th instance timed and scaled), both
      with the long run's budget; instances that miss it within the budget are counted as
      censored, not as reached."""
    import pimqap
    b0, ratio = ladder
    M = max(1, budget // 4)

    def params(seed, **kw):
        return pimqap.default_params(replicas=replicas, groups=1, sweeps_per_exchange=4, beta_max=b0,
                                     beta_ratio=ratio, beta_internal=1, seed=seed, **kw)

    pairs = [(b.F, b.D) for b in batch]
    props = sum(_sweeps_proposals(b.n, replicas, 4 * M) for b in batch)
    pimqap.batch_solve(pairs[:2], [params(1, max_megaiters=2), params(2, max_megaiters=2)])   # warm-up
    t0 = time.perf_counter()
    tuning = pimqap.batch_tune(pairs, [params(k + 1, max_megaiters=M) for k in range(len(batch))])
    tune_wall = time.perf_counter() - t0

    def fixed_work(autotune):
        os.environ["PIMQAP_AUTOTUNE"] = "1" if autotune else "0"
        try:
            t0 = time.perf_counter()
            res = pimqap.batch_solve(pairs, [params(k + 1, max_megaiters=M) for k in range(len(batch))])
            return time.perf_counter() - t0, res
        finally:
            os.environ.pop("PIMQAP_AUTOTUNE", None)

    rules_wall, _ = fixed_work(False)
    fixed_wall, fixed = fixed_work(True)
    if args.batch_fixed_only:   # the fixed-work batch alone (profiling)
        print(json.dumps({"suite": name, "instances": len(batch), "sweeps": 4 * M, "wall_s": fixed_wall,
                          "proposals_per_s_wall": props / fixed_wall, "fixed_rules_wall_s": rules_wall}))
        return
    t0 = time.perf_counter()
    longrun = pimqap.batch_solve(pairs, [params(10 ** 6 + k, max_megaiters=4 * M) for k in range(len(batch))])
    long_wall = time.perf_counter() - t0
    targets = [min(l["best_energy"], f["best_energy"]) for l, f in zip(longrun, fixed)]
    goals = [int(t + abs(t) // 1000) for t in targets]          # gap <= 0.1 %
    checks = []
    for k in range(0, len(batch), max(1, len(batch) // max(1, xcheck)))[:xcheck]:
        got = _ref_best(batch[k].F, batch[k].D, replicas, args.xcheck_sweeps, b0, ratio)
        if got:
            got.update(instance=k, n=batch[k].n, target=targets[k],
                       target_at_or_below_reference=targets[k] <= got["best"])
            checks.append(got)
    t0 = time.perf_counter()
    res = pimqap.batch_solve(pairs, [params(k + 1, max_megaiters=4 * M, goal=goals[k]) for k in range(len(batch))])
    batch_ttt = time.perf_counter() - t0
    reached = sum(1 for r in res if r["stopped_by"] == 1)
    ttt_each = sorted(r["time_to_target_ms"] for r in res if r["stopped_by"] == 1)
    sample = list(range(0, len(batch), plain_every))
    t0 = time.perf_counter()
    plain_reached = 0
    for k in sample:
        r = pimqap.solve(batch[k].F, batch[k].D, params(k + 1, max_megaiters=4 * M, goal=goals[k]))
        plain_reached += r["stopped_by"] == 1
    plain_sample = time.perf_counter() - t0
    plain_total = plain_sample * len(batch) / len(sample)
    line = {"suite": name, "metric": "time-to-target (<=0.1% gap) and swap proposals/sec",
            "instances": len(batch), "n_range": [min(b.n for b in batch), max(b.n for b in batch)],
            "replicas": replicas, "sweeps": 4 * M,
            "ladder": {"beta0_internal": b0, "beta_ratio": ratio},
            "autotuner": {"wall_s": tune_wall, "classes": tuning},
            "fixed_work": {"wall_s": fixed_wall, "proposals_per_s_wall": props / fixed_wall,
                           "fixed_rules_wall_s": rules_wall, "fixed_rules_proposals_per_s_wall": props / rules_wall,
                           "accept_rate": sum(r["accepts"] for r in fixed) / sum(r["updates"] for r in fixed)},
            "targets": f"best of a {16 * M}-sweep batch run (other seeds) and the {4 * M}-sweep run; "
                       f"goal = target + |target| // 1000",
            "long_run_wall_s": long_wall,
            "reference_cross_check": checks,
            "ttt_budget_sweeps": 16 * M,
            "batch_time_to_target_s": batch_ttt, "batch_reached": reached,
            "batch_censored": len(batch) - reached,
            "batch_ttt_ms_p50_p90_of_reached": [ttt_each[len(ttt_each) // 2], ttt_each[int(0.9 * len(ttt_each))]]
            if ttt_each else None,
            "plain_time_to_target_s_est": plain_total, "plain_sampled": len(sample),
            "plain_reached_in_sample": plain_reached,
            "speedup_vs_plain": plain_total / batch_ttt}
    print(json.dumps(line))


def run_batch_suite(args):
    """512 instances, n ~ U[20, 150], uniform [0, 99] flows and distances, 32 replicas each,
    2000 sweeps, in persistent launches (run_ttt_suite)."""
    batch = instances.uniform_batch(args.batch_instances)
    run_ttt_suite(args, "batch", batch, 32, LADDER_UNIFORM, args.batch_sweeps, 16, args.xcheck)


def run_heavy_suite(args):
    """128 heavy-tailed instances, n ~ U[100, 256] (lognormal flows with 70 % zeros, Euclidean
    distances), 64 replicas each, int64 energies (run_ttt_suite)."""
    batch = instances.heavy_batch(args.heavy_instances)
    run_ttt_suite(args, "heavy", batch, 64, LADDER_HEAVY, args.heavy_sweeps, 8, args.xcheck)


def _serve_params(pimqap, inst, k):
    b0, ratio = LADDER_UNIFORM if inst.name.startswith("uniform") else LADDER_HEAVY
    return pimqap.default_params(replicas=32, groups=1, sweeps_per_exchange=4, beta_max=b0,
                                 beta_ratio=ratio, beta_internal=1, seed=k + 1, max_megaiters=500)


def serve_once(rate, duration, drain):
    """One Poisson trace (`rate` arrivals/s for `duration` s) into a fresh server; results are
    collected for up to `drain` s after the last arrival.  The request sequence (instances and
    seeds) is the same at every rate; only the arrival times scale."""
    import pimqap
    trace = list(instances.serving_trace(rate_hz=rate, duration_s=duration))
    # the autotuner's sample: 64 requests spread over the trace (it picks classes and SM shares
    # from them; shapes it misses still get a launch of their own)
    step = max(1, len(trace) // 64)
    sample = [(inst.F, inst.D, _serve_params(pimqap, inst, k)) for k, (_, inst) in enumerate(trace)
              if k % step == 0][:64]
    srv = pimqap.Server(sample=sample)
    t_start = time.perf_counter()
    tickets = []
    done = {}
    failure = None
    try:
        for k, (t_arr, inst) in enumerate(trace):
            now = time.perf_counter() - t_start
            if t_arr > now:
                time.sleep(t_arr - now)
            tickets.append((srv.submit(inst.F, inst.D, _serve_params(pimqap, inst, k)), k, inst))
        deadline = t_start + duration + drain
        while len(done) < len(tickets) and time.perf_counter() < deadline:
            for t, k, inst in tickets:
                if t in done:
                    continue
                r = srv.poll(t)
                if r is not None:
                    done[t] = (r, k, inst, time.perf_counter() - t_start)
            time.sleep(0.01)
    except pimqap.PimqapError as e:   # the run ends; its row says why
        failure = f"{e} (after {time.perf_counter() - t_start:.1f} s, {len(tickets)} submitted)"
    st = srv.stats()
    srv.close()
    lat = sorted(r["latency_ms"] for r, _, _, _ in done.values())
    t_last = max((t for _, _, _, t in done.values()), default=0.0)
    props = sum(_sweeps_proposals(inst.n, 32, r["megaiters_done"] * 4) for r, _, inst, _ in done.values())

    def pct(q):
        return lat[min(len(lat) - 1, int(q * len(lat)))] if lat else None

    row = {"rate_hz": rate, "duration_s": duration, "submitted": len(tickets), "completed": len(done),
           "backlog_at_end": len(tickets) - len(done), "p50_ms": pct(0.50), "p99_ms": pct(0.99),
           "max_ms": lat[-1] if lat else None,
           "throughput_req_per_s": len(done) / t_last if t_last else 0.0,
           "proposals_per_s": props / t_last if t_last else 0.0,
           "admitted": st["admitted"], "classes": st["classes"], "error_word": st["error_word"],
           "failure": failure}
    return row, {k: (r, inst) for r, k, inst, _ in done.values()}


def run_serve_suite(args):
    """Serving at the published load: Poisson arrivals of QAP solves, n ~ U[30, 256], half
    uniform, half heavy-tailed instances, 32 replicas and 2000 sweeps each, into the
    continuous-batching server, for --duration s.  A search over --rates finds the highest rate
    whose p99 latency stays within --p99-bound s with no backlog; that rate and --rate (the
    published 200 req/s) are reported with p50 / p99 latency, throughput, backlog and each
    completed request's gap to its best-known cost (the best of a batch run four times as long,
    other seeds)."""
    import pimqap
    rows = []
    results = {}
    for rate in [float(r) for r in args.rates.split(",") if r]:
        row, got = serve_once(rate, args.duration, args.drain)
        rows.append(row)
        results[rate] = got
    ok = [r for r in rows if r["backlog_at_end"] == 0 and r["p99_ms"] is not None and not r["failure"]
          and r["p99_ms"] <= 1e3 * args.p99_bound]
    best = max(ok, key=lambda r: r["rate_hz"]) if ok else None
    over, got_over = serve_once(args.rate, args.duration, args.drain)
    # best-known costs of every request that completed in either run
    ks = sorted(set(k for rate in ([best["rate_hz"]] if best else []) for k in results[rate]) | set(got_over))
    trace = list(instances.serving_trace(rate_hz=args.rate, duration_s=args.duration))
    if best:
        trace_b = list(instances.serving_trace(rate_hz=best["rate_hz"], duration_s=args.duration))
        trace = trace if len(trace) >= len(trace_b) else trace_b
    insts = {k: trace[k][1] for k in ks if k < len(trace)}
    t0 = time.perf_counter()
    order = sorted(insts)
    lparams = []
    for k in order:                      # four times the sweeps, another seed
        p = _serve_params(pimqap, insts[k], 10 ** 6 + k)
        p.max_megaiters = 4 * p.max_megaiters
        lparams.append(p)
    long = pimqap.batch_solve([(insts[k].F, insts[k].D) for k in order], lparams) if order else []
    targets = {k: r["best_energy"] for k, r in zip(order, long)}
    long_wall = time.perf_counter() - t0

    def gaps(got):
        g = []
        for k, (r, inst) in got.items():
            t = min(targets.get(k, r["best_energy"]), r["best_energy"])
            g.append((r["best_energy"] - t) / abs(t) if t else 0.0)
        g.sort()
        if not g:
            return None
        return {"requests": len(g), "median": g[len(g) // 2], "p90": g[int(0.9 * len(g))], "max": g[-1],
                "within_0.1pct": sum(1 for x in g if x <= 1e-3) / len(g),
                "within_1pct": sum(1 for x in g if x <= 1e-2) / len(g)}

    if best:
        best = dict(best, gap=gaps(results[best["rate_hz"]]))
    over = dict(over, gap=gaps(got_over))
    line = {"suite": "serve", "metric": "serve p50/p99 latency, throughput and gap to best-known",
            "requests": "n ~ U[30, 256], half uniform [0, 99], half heavy-tailed; 32 replicas, 2000 sweeps",
            "duration_s": args.duration, "drain_s": args.drain, "p99_bound_s": args.p99_bound,
            "rate_search": rows, "sustainable": best, "published_rate": over,
            "best_known": "best of a batch run of the same request with 4x the sweeps (other seed)",
            "best_known_wall_s": long_wall}
    print(json.dumps(line))


def run_divergence_suite(args):
    """Decision divergence between the GPU kernel (fp64 exp2 weights, tree-ordered fp64 sums) and
    the reference's arithmetic (x87 exp2l weights, sequential long-double sums rounded to double,
    CPU_PIM.cpp:236-251) as restated by the oracle, on the headline workload (n = 256 grid
    instance, 64 replicas, exchange every 4 sweeps) at the benchmark's ladder and at a hot
    ladder.  Both sides run the same Philox stream in lock step; every --div-chunk
    mega-iterations the permutation, energy and best energy of every replica are compared.  Any differing decision changes a permutation at once, so the first mismatching
    chunk bounds the first divergence; a run then ends and the next starts from a new seed.
    Reports the updates compared and the divergences seen."""
    import pimqap
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle
    orc = Oracle()
    inst = instances.grid256(1000)
    ladders = {"bench": (BETA_MAX, BETA_RATIO), "hot": (2.0 ** -10, BETA_RATIO)}
    per_ladder = args.div_updates
    out = {"suite": "divergence", "workload": "grid256 n=256, 64 replicas, exchange every 4 sweeps",
           "chunk_megaiters": args.div_chunk, "ladders": {}}
    t_start = time.perf_counter()
    for name, (b0, ratio) in ladders.items():
        done, divergences, runs, first = 0, 0, 0, []
        seed = 1
        while done < per_ladder:
            runs += 1
            p = pimqap.default_params(replicas=REPLICAS, groups=1, sweeps_per_exchange=SWEEPS_PER_EXCHANGE,
                                      beta_max=b0, beta_ratio=ratio, beta_internal=1, seed=seed,
                                      max_megaiters=2 ** 31 - 1, megaiters_per_launch=args.div_chunk)
            st = orc.setup(inst.D, inst.F, 1, REPLICAS, SWEEPS_PER_EXCHANGE, b0, ratio, seed, cap=REPLICAS)
            with pimqap.Solver(inst.F, inst.D, p) as s:
                m = 0
                while done < per_ladder:
                    s.run(args.div_chunk)
                    orc.run(st, inst.D, inst.F, args.div_chunk, -(1 << 62))
                    m += args.div_chunk
                    # permutation, energy and best of every replica slot (the exchange the solver
                    # runs at the end of a launch moves betas, not these)
                    bad = False
                    for l in range(REPLICAS):
                        r = s.replica(0, l, force=False)
                        if (not np.array_equal(r["phi"], st.phi[0, l]) or r["E"] != st.E[0, l]
                                or r["bestE"] != st.bestE[0, l]):
                            bad = True
                            break
                    if bad:
                        divergences += 1
                        first.append({"seed": seed, "megaiter_chunk_end": m})
                        break
                    done += REPLICAS * SWEEPS_PER_EXCHANGE * args.div_chunk * N
            seed += 1
        out["ladders"][name] = {"beta0_internal": b0, "beta_ratio": ratio, "updates_compared": done,
                                "divergences": divergences, "runs": runs, "divergent_chunks": first,
                                "rate_upper_95": 3.0 / done if divergences == 0 else None}
    out["wall_s"] = time.perf_counter() - t_start
    print(json.dumps(out))


def run_oneshot_divergence_suite(args):
    """Decision divergence of the one-shot rule between the solver's kernel and GPU-CUPIM's own
    kernels (perl-gpu/src/lib/qap/qap.cu:1462-1600, built from the reference source into
    oracle/_ref/libref_cupim.so with its cuRANDDx generator replaced by one that copies the
    solver's thresholds), for both of the solver's weight functions: CUDA's exp2f as the
    reference writes it (oneshot_weights 0, the default) and the library's own 2^x
    (oneshot_weights 1, the one the oracle restates).  Headline instance;
    64 groups of one replica each (rank_slots 1: no exchange moves a beta), so the reference's
    pool of 64 replicas takes exactly the solver's steps; a cold, a middle and a hot beta.  Every
    --div-chunk mega-iterations (4 steps each) the permutation and energy of every replica are
    compared; on a mismatch the divergence is counted and the reference's pool is reset to the
    solver's permutations (its force matrices recomputed from them) and the run goes on.
    Reports the proposals compared and the divergences seen."""
    import tempfile
    import pimqap
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import CupimRef, Oracle
    orc = Oracle()
    ref = CupimRef()
    inst = instances.grid256(1000)
    G, spe = REPLICAS, SWEEPS_PER_EXCHANGE
    betas = {"cold": BETA_MAX, "middle": BETA_MAX / 8, "hot": BETA_MAX / 64}
    out = {"suite": "divergence", "update_rule": "one-shot",
           "workload": "grid256 n=256, 64 groups of one replica (no exchange), 4 steps per mega-iteration",
           "reference": "GPU-CUPIM os_* kernels built from the reference source (oracle/_ref/libref_cupim.so)",
           "chunk_megaiters": args.div_chunk, "betas": {}}
    t_start = time.perf_counter()
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "grid256.dat")
        instances.write_instance(path, inst)
        for (wname, weights), (name, beta) in [(w, b) for w in (("cuda_exp2f", 0), ("own_exp2", 1))
                                                for b in betas.items()]:
            seed = 7
            p = pimqap.default_params(replicas=1, groups=G, rank_slots=1, sweeps_per_exchange=spe,
                                      beta_max=beta, beta_ratio=1.5, beta_internal=1, seed=seed,
                                      max_megaiters=2 ** 31 - 1, megaiters_per_launch=args.div_chunk,
                                      update_rule=pimqap.RULE_ONE_SHOT, goal=-(1 << 62),
                                      oneshot_weights=weights)
            bvec = np.full(G, np.float32(beta), np.float32)
            done, divergences, first, swaps_seen = 0, 0, [], 0
            ref.open(path, G)
            try:
                with pimqap.Solver(inst.F, inst.D, p) as s:
                    phi = np.stack([s.replica(g, 0, force=False)["phi"] for g in range(G)]).astype(np.int32)
                    ref.set(phi, bvec)
                    step = 0
                    while done < args.div_updates:
                        s.run(args.div_chunk)
                        for _ in range(args.div_chunk * spe):
                            ref.step(orc.oneshot_uniforms(seed, G, 1, step, N))
                            step += 1
                        cphi, _, cscore, _ = ref.get(force=False)
                        mine = [s.replica(g, 0, force=False) for g in range(G)]
                        sphi = np.stack([r["phi"] for r in mine])
                        swaps_seen += int(np.count_nonzero(sphi != phi))
                        bad = [g for g in range(G) if not np.array_equal(mine[g]["phi"], cphi[g])
                               or mine[g]["E"] != int(cscore[g])]
                        done += G * args.div_chunk * spe * N
                        if bad:
                            divergences += 1
                            first.append({"step_chunk_end": step, "groups": bad[:8]})
                            ref.set(sphi, bvec)
                        phi = sphi
            finally:
                ref.close()
            out["betas"][f"{wname}/{name}"] = {"beta_internal": beta, "oneshot_weights": weights, "proposals_compared": done, "divergent_chunks": divergences,
                                  "first": first[:10], "locations_moved_per_chunk":
                                  swaps_seen / max(1, done // (G * args.div_chunk * spe * N)),
                                  "rate_upper_95": 3.0 / done if divergences == 0 else None}
    out["wall_s"] = time.perf_counter() - t_start
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="grid256",
                    help="headline instance (clique92: the tai256c program's structure and moves; "
                         "cfg1: n=32, 16 replicas, exchange every sweep)")
    ap.add_argument("--groups", type=int, default=1,
                    help="independent parallel-tempering groups of the workload's replicas per GPU (the "
                         "reference's -t; its CPU arm runs one group per host thread)")
    ap.add_argument("--pipeline", type=int, default=0, choices=[0, 1, 2],
                    help="binary-flow kernel: 2 = the pipelined epoch (next update's deltas during the pick)")
    ap.add_argument("--tensor-update", type=int, default=0, choices=[0, 1, 2, 3],
                    help="one-shot rule's force update: 0 = automatic, 1 = integer CUDA cores, "
                         "2 = mma.sync, 3 = tcgen05 (tensor memory)")
    ap.add_argument("--launch-mode", type=int, default=0, choices=[0, 1, 2],
                    help="0 = automatic (persistent when resident), 1 = a launch per mega-iteration, 2 = persistent")
    ap.add_argument("--update-rule", choices=["sequential", "one-shot"], default="sequential",
                    help="sequential: CPU_PIM's sweeps (the headline); one-shot: GPU-CUPIM's parallel step")
    ap.add_argument("--cluster-size", type=int, default=0, help="CTAs per replica (0 = automatic)")
    ap.add_argument("--threads", type=int, default=0, help="threads per replica and CTA (0 = automatic)")
    ap.add_argument("--pairing", type=int, default=0, choices=[0, 1, 2],
                    help="replicas per CTA set of the binary-flow kernel: 0 = automatic, 1, 2")
    ap.add_argument("--suite", choices=["headline", "batch", "heavy", "serve", "divergence"], default="headline",
                    help="headline: the n=256 workload (the driver's line); batch / serve: the other "
                         "workloads; divergence: GPU vs oracle decisions over a long stream (with "
                         "--update-rule one-shot: GPU vs the reference's own one-shot kernels)")
    ap.add_argument("--div-updates", type=int, default=10_000_000,
                    help="divergence suite: updates compared per ladder")
    ap.add_argument("--div-chunk", type=int, default=10, help="divergence suite: mega-iterations per comparison")
    ap.add_argument("--batch-instances", type=int, default=512, help="batch suite: instances")
    ap.add_argument("--batch-sweeps", type=int, default=2000, help="batch suite: sweeps per instance")
    ap.add_argument("--batch-fixed-only", action="store_true",
                    help="batch / heavy suites: run only the fixed-work batch (profiling)")
    ap.add_argument("--heavy-instances", type=int, default=128, help="heavy suite: instances")
    ap.add_argument("--heavy-sweeps", type=int, default=1000, help="heavy suite: sweeps per instance")
    ap.add_argument("--xcheck", type=int, default=4,
                    help="batch / heavy suites: instances whose targets are checked against the reference's CPU code")
    ap.add_argument("--xcheck-sweeps", type=int, default=2000,
                    help="batch / heavy suites: sweeps of each reference group in that check (capped at 120 s)")
    ap.add_argument("--rate", type=float, default=200.0, help="serve suite: the published arrival rate (req/s)")
    ap.add_argument("--rates", default="2,3,4,5", help="serve suite: arrival rates searched for the highest "
                                                     "sustainable one (comma separated)")
    ap.add_argument("--p99-bound", type=float, default=10.0, help="serve suite: p99 latency bound (s)")
    ap.add_argument("--duration", type=float, default=60.0, help="serve suite: seconds of arrivals")
    ap.add_argument("--drain", type=float, default=60.0, help="serve suite: seconds allowed after arrivals end")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.suite == "batch":
        run_batch_suite(args)
        return
    if args.suite == "heavy":
        run_heavy_suite(args)
        return
    if args.suite == "serve":
        run_serve_suite(args)
        return
    if args.suite == "divergence":
        if args.update_rule == "one-shot":
            run_oneshot_divergence_suite(args)
        else:
            run_divergence_suite(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
