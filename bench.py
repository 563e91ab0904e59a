"""Benchmark: the fused radix partition -> unique-build hash join -> dense
group-by of the 150M-row build x 600M-row probe workload on one B200
(SELECT group, SUM(price*(100-disc)), COUNT(*) ... GROUP BY group over 1.5M
groups), reported as join+agg rows/s = (build rows + probe rows) / s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step is one full pass over resident inputs: partition both sides, build
and probe every round, aggregate, and compact the occupied groups (one host
wait for the bucket counts, one for the group count).  Under torchrun each
rank runs an independent replica of the workload on its own GPU (the path is
replicas-only across GPUs); the time is the max over ranks.

The JSON line also carries: the dominant kernel's live roofline (algorithmic
bytes per launch / CUDA-event launch time, against the measured HBM copy
bandwidth), the whole step's, the end-to-end rate through the public API with
host buffers and host<->device copies inside the timed region, the oracle's
CPU rate on a bounded sample, the SM clocks sampled during the timed region,
and the number of this library's kernels launched in it.  ``--impl
reference`` times the reference algorithm's CPU restatement (the oracle) on
all host threads instead.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FALLBACK_HBM_GBS = 6650.0


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="scale",
                    help="scale (150M x 600M), small (250K x 1M) or scale/<divisor>")
    ap.add_argument("--B", type=int, default=0, help="fan-out (0: the autotuner's pick)")
    ap.add_argument("--parallelism", choices=["sharded", "replicas"], default=None,
                    help="one join sharded over the ranks (each holds a slice of both sides; "
                         "buckets move to their owners; the default for N > 1) or independent "
                         "replicas (the default for N = 1)")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain-form", action="store_true",
                    help="skip timing the reference's own GPU path")
    ap.add_argument("--plain-steps", type=int, default=5)
    ap.add_argument("--batch-gb", type=float, default=60.0,
                    help="batch workload: device bytes of one wave")
    ap.add_argument("--plain-instances", type=int, default=0,
                    help="batch workload: instances the reference path runs (0: the whole wave)")
    ap.add_argument("--cpu-sample", type=float, default=0.01,
                    help="fraction of the workload the CPU baseline joins per sample")
    ap.add_argument("--serve-requests", type=int, default=400,
                    help="serve workload: requests in the trace")
    ap.add_argument("--serve-rates", default="50,100,200,400,800,1200,1600,2000",
                    help="serve workload: offered rates (requests/s) of the sweep")
    ap.add_argument("--serve-iter-rows", type=int, default=1 << 27,
                    help="serve workload: probe rows one persistent launch takes")
    return ap.parse_args(argv)


def workload(name: str):
    from pageflow_b200 import datagen
    if name == "scale":
        return datagen.SCALE
    if name == "small":
        return datagen.SMALL
    if name.startswith("scale/"):
        return datagen.scaled(datagen.SCALE, 1 / float(name.split("/", 1)[1]))
    raise SystemExit(f"unknown workload {name}")


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---- replicas ----------------------------------------------------------------------

def max_over_ranks(ms: float, world: int, device) -> float:
    """The job's time: the slowest rank's (every rank runs its own replica)."""
    if world == 1:
        return float(ms)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int, device) -> float:
    """The sum of a per-rank quantity over the ranks."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(units_per_rank: float, ms: float, world: int) -> float:
    """Whole-job throughput: the units all ranks processed over the job's
    time (weak scaling: each rank processes units_per_rank)."""
    return world * units_per_rank / (ms / 1e3)


# ---- clocks -------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi samples of this GPU's clocks every 100 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        cmd = ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
               "-lms", "100"]
        if gpu_id:
            cmd += ["-i", gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if r[5 + i].lower() in ("active", "1", "yes")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ---- the reference arm / CPU baseline -------------------------------------------

def cpu_sample_run(w, frac: float, reps_seconds: float = 10.0):
    """The oracle's join + group-by (the reference algorithm restated in C,
    partitioned by mix64 and joined by sort + binary search on every host
    thread) on a bounded sample of the workload: `frac` of its rows, repeated
    for about `reps_seconds`.  Returns (rows/s, threads, description)."""
    import oracle
    oracle.build()
    nb = max(1, int(w.n_build * frac))
    npr = max(1, int(w.n_probe * frac))
    ng = max(1, int(w.n_groups * frac))
    bkey, bgrp = oracle.gen_build(w.seed, nb, ng)
    fk, price, disc = oracle.gen_probe(w.config, w.seed, nb, 0, npr)
    threads = oracle.threads()
    runs, t0 = 0, time.perf_counter()
    while True:
        oracle.join_aggregate(bkey, bgrp, fk, price, disc, w.scale, 0, ng, B=256,
                              n_threads=threads)
        runs += 1
        el = time.perf_counter() - t0
        if el >= reps_seconds or runs >= 50:
            break
    rate = (nb + npr) * runs / el
    desc = (f"{nb} build x {npr} probe rows ({frac:g} of the workload, {ng} groups), "
            f"{runs} runs in {el:.1f} s")
    return rate, threads, desc


def run_reference(args, w, world, rank):
    if rank != 0:
        return
    import oracle
    oracle.build()
    frac = args.cpu_sample
    nb = max(1, int(w.n_build * frac))
    npr = max(1, int(w.n_probe * frac))
    ng = max(1, int(w.n_groups * frac))
    bkey, bgrp = oracle.gen_build(w.seed, nb, ng)
    fk, price, disc = oracle.gen_probe(w.config, w.seed, nb, 0, npr)
    threads = oracle.threads()
    for _ in range(args.warmup):
        oracle.join_aggregate(bkey, bgrp, fk, price, disc, w.scale, 0, ng, B=256,
                              n_threads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.join_aggregate(bkey, bgrp, fk, price, disc, w.scale, 0, ng, B=256,
                              n_threads=threads)
    el = time.perf_counter() - t0
    rate = (nb + npr) * args.steps / el
    sample = (f"{nb} build x {npr} probe rows per step ({frac:g} of the workload, {ng} "
              f"groups)")
    line = {
        "impl": "reference", "metric": "join+agg rows/s", "value": rate, "unit": "rows/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": w.name, "build_rows": w.n_build, "probe_rows": w.n_probe,
                   "groups": w.n_groups, "parallelism": "replicas"},
        "cpu_baseline": {"value": rate, "unit": "rows/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": rate, "unit": "rows/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- ours ------------------------------------------------------------------------------

def algorithmic_bytes(w, B_rounds):
    """Algorithmic DRAM bytes per step, per kernel (name -> bytes): the
    columns each pass must read and write once.  k_fhist reads each side's
    keys; the scatters read the source columns and write the carried ones
    (build: key 8 + group 4; probe: fk 8 + value 8, from fk, price and
    discount).  Shared-memory path: k_p2_hist reads both sides' keys, the
    second scatter reads and writes the carried columns (build 12 + 12,
    probe 16 + 16 a row), k_sjoin reads the sub-partitioned sides once
    (build 12 B, probe 16 B a row).  L2-round path: k_fround (build round
    r + 1 while probing round r) reads the partitioned sides once.  The
    finish reads the 16-byte slab and writes the groups it keeps.  A step
    counts the kernels it ran."""
    nb, npr, g = w.n_build, w.n_probe, w.n_groups
    return {
        "k_fhist": 8 * (nb + npr),          # counted passes only
        "k_fscatter_build": nb * (12 + 12),
        "k_fscatter_probe": npr * (24 + 16),
        "k_p2_hist": 8 * (nb + npr),        # counted passes only
        "k_p2_scatter": nb * (12 + 12) + npr * (16 + 16),
        "k_sjoin": nb * 12 + npr * 16,
        "k_fround": nb * 12 + npr * 16,
        "k_gcount": g * 8,
        "k_gemit": g * 16 + g * 24,
    }


def run_ours(args, w, world, rank, local_rank):
    import torch
    import torch.distributed as dist

    from pageflow_b200 import _native, datagen
    from pageflow_b200.join_aggregate import JoinAggregate

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    bkey, bgrp = datagen.gen_build(w, dev)
    fk, price, disc = datagen.gen_probe(w, dev)
    plan = JoinAggregate(w.n_build, w.n_probe, 0, w.n_groups, dev, B=args.B or None,
                         scale=w.scale)
    torch.cuda.synchronize()

    def step():
        plan.aggregate(bkey, bgrp, fk, price, disc)
        return plan.finish()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    keys, sums, counts = step()
    n_groups_out = int(keys.numel())
    matched = plan.read_stats().matched
    # the autotuner's pick (made on the first warm-up call) and its timings
    tuning = None
    if plan.tuning is not None:
        t = plan.tuning
        tuning = {"choice": {"B": t.choice.B, "table": t.choice.table,
                             "sub_rows": t.choice.sub_rows, "counted": t.choice.counted},
                  "cached": t.cached, "candidate_ms": t.times_ms}
    elif plan.knobs is None:
        tuning = {"off": "a PF_* override or an explicit --B fixes the configuration"}
    # rounds of the plan (for the per-launch figures)

    gpu_id = None
    try:
        gpu_id = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    sampler = ClockSampler(gpu_id)
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = _native.launch_count()
    _native.profile_begin()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    prof = _native.profile_end()
    launches = _native.launch_count() - launches0
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
    rows_step = w.n_build + w.n_probe
    value = job_rate(rows_step * args.steps, ms, world)

    # roofline: the dominant kernel's live figure and the whole step's
    peak, peak_kind = measured_peak()
    alg = algorithmic_bytes(w, None)
    dom = max(prof.items(), key=lambda kv: kv[1][0]) if prof else None
    roofline = None
    kernels = {}
    for name, (tot_ms, n) in sorted(prof.items(), key=lambda kv: -kv[1][0]):
        per_step_launches = n / args.steps
        entry = {"ms_per_step": tot_ms / args.steps, "launches_per_step": per_step_launches,
                 "share": None}
        if name in alg and tot_ms > 0:
            entry["gbs"] = alg[name] * args.steps / (tot_ms / 1e3) / 1e9
        kernels[name] = entry
    tot_kernel_ms = sum(v[0] for v in prof.values()) or 1.0
    for name in kernels:
        kernels[name]["share"] = prof[name][0] / tot_kernel_ms
    if dom is not None:
        name, (tot_ms, n) = dom
        bytes_launch = alg.get(name, 0) * args.steps / n
        avg_s = tot_ms / n / 1e3
        achieved = bytes_launch / avg_s / 1e9
        traffic = None
        tfile = ROOT / "profiles" / "traffic.json"
        if tfile.exists():
            try:
                tj = json.loads(tfile.read_text())
                if tj.get("workload") == w.name and name in tj.get("kernels", {}):
                    traffic = tj["kernels"][name]["dram_bytes_per_launch"]
            except Exception:
                traffic = None
        roofline = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak,
                    "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                    "bytes_per_launch": bytes_launch, "peak_source": peak_kind}
    step_bytes = sum(b for name, b in alg.items() if name in prof)
    step_gbs = step_bytes / (ms / args.steps / 1e3) / 1e9
    # the same step against the bytes a two-pass radix join + group-by must
    # move whatever its kernels: each side read once and its carried columns
    # written and read once a pass, the groups once
    # (sum over sides of N * (w_in + 2 * P * w_c) + G * (4 + 16), P = 2)
    formula = (w.n_build * (12 + 4 * 12) + w.n_probe * (24 + 4 * 16) + w.n_groups * 20)
    formula_gbs = formula / (ms / args.steps / 1e3) / 1e9
    step_roofline = {"bound": "hbm", "algorithmic_bytes": step_bytes, "achieved": step_gbs,
                     "peak": peak, "unit": "GB/s", "frac": step_gbs / peak,
                     "peak_source": peak_kind,
                     "two_pass_bytes": formula, "two_pass_achieved": formula_gbs,
                     "two_pass_frac": formula_gbs / peak}

    # end to end through the public API, host buffers
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, w, plan, dev, (bkey, bgrp, fk, price, disc), world)

    plain = None
    if not args.no_plain_form:
        plain = run_plain_form(args, w, dev, (bkey, bgrp, fk, price, disc), keys, sums, counts,
                               ms / args.steps)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, threads, desc = cpu_sample_run(w, args.cpu_sample)
        cpu = {"value": rate, "unit": "rows/s", "cores": threads, "kind": "port",
               "sample": desc}

    if rank == 0:
        line = {
            "metric": "join+agg rows/s", "value": value, "unit": "rows/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int64", "data": "synthetic (seeded generator, inputs on the device)",
            "config": {"workload": w.name, "build_rows": w.n_build, "probe_rows": w.n_probe,
                       "groups": w.n_groups, "fanout_B": plan.B, "parallelism":
                       "replicas" if world > 1 else "single",
                       "l2": "inputs (16 B/row build, 24 B/row probe) exceed L2; no flush",
                       "groups_out": n_groups_out, "matched_probe_rows": matched,
                       "autotune": tuning},
            "roofline": roofline, "step_roofline": step_roofline,
            "kernels": kernels,
            "e2e": e2e, "cpu_baseline": cpu, "plain_form": plain, "clocks": clocks,
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)


def run_sharded(args, w, world, rank, local_rank):
    """N > 1: one join over the ranks (weak scaling: every rank holds the
    scale workload's rows, so the job joins N x 150M build rows with N x 600M
    probe rows, keys permuted over all N x 150M).  A step: each rank
    partitions its rows (pf_join_partition), sends every bucket to its owner
    over NCCL point-to-point messages, joins the buckets it owns
    (pf_join_aggregate_buckets) and the ranks add their group slabs (an
    int64 all-reduce).  Device time, max over ranks."""
    import dataclasses

    import torch
    import torch.distributed as dist

    from pageflow_b200 import _native, datagen
    from pageflow_b200.sharded import CudaPhases, ShardedJoinAggregate, dense_groups

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    g = dataclasses.replace(w, n_build=w.n_build * world, n_probe=w.n_probe * world)
    bkey, bgrp = datagen.gen_build(g, dev, lo=rank * w.n_build, rows=w.n_build)
    fk, price, disc = datagen.gen_probe(g, dev, lo=rank * w.n_probe, rows=w.n_probe)
    B = args.B or max(256, world)
    job = ShardedJoinAggregate(0, w.n_groups, B, scale=w.scale, phases=CudaPhases(dev))
    for _ in range(args.warmup):
        job.run(bkey, bgrp, fk, price, disc)
    sums, counts = job.run(bkey, bgrp, fk, price, disc)
    keys, _, _ = dense_groups(sums, counts, 0)
    groups_out, matched = int(keys.numel()), int(counts.sum())
    sampler = ClockSampler(None)
    dist.barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = _native.launch_count()
    e0.record(stream)
    for _ in range(args.steps):
        job.run(bkey, bgrp, fk, price, disc)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = _native.launch_count() - launches0
    dist.barrier()
    clocks = sampler.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
    rows_step = w.n_build + w.n_probe
    value = job_rate(rows_step * args.steps, ms, world)
    # end to end: every rank's inputs from pinned host memory each step, the
    # dense groups back to the host
    e2e = None
    if not args.no_e2e:
        host = [t.cpu().pin_memory() for t in (bkey, bgrp, fk, price, disc)]
        dev_in = [bkey, bgrp, fk, price, disc]
        h2d = sum(t.numel() * t.element_size() for t in host)

        def e2e_step():
            for d, h in zip(dev_in, host):
                d.copy_(h, non_blocking=True)
            su, co = job.run(*dev_in)
            out = [su.to("cpu", non_blocking=True), co.to("cpu", non_blocking=True)]
            return out, su.numel() * 16
        e2e_step()
        torch.cuda.synchronize()
        dist.barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        d2h = 0
        for _ in range(args.e2e_steps):
            _, d2h = e2e_step()
        f1.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(f0.elapsed_time(f1), world, dev)
        e2e = {"value": job_rate(rows_step * args.e2e_steps, ems, world), "unit": "rows/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": ems / args.e2e_steps}
    moved = sum_over_ranks(sum(job.last["received_rows"]) - sum(job.last["kept_rows"]),
                           world, dev)
    # per rank: the bytes the step must move in HBM (counts, the partition
    # pass, the exchange's writes of every received or kept row and reads of
    # every sent one, the second pass and the join, as on one GPU) and over
    # NVLink (the rows this rank received from its peers, the slowest rank's)
    nb, npr = w.n_build, w.n_probe
    recv = [job.last["received_rows"][s] - job.last["kept_rows"][s] for s in range(2)]
    link_bytes = max_over_ranks(float(recv[0] * 12 + recv[1] * 16), world, dev)
    hbm_bytes = (8 * (nb + npr) + nb * 24 + npr * 40 + 2 * (nb * 12 + npr * 16)
                 + nb * 24 + npr * 32 + nb * 12 + npr * 16)
    peak, peak_src = measured_peak()
    step_s = ms / args.steps / 1e3
    roof = {"bound": "hbm", "kernel": "step, per rank (partition, exchange, second pass, join)",
            "achieved": hbm_bytes / step_s / 1e9, "peak": peak, "unit": "GB/s",
            "frac": hbm_bytes / step_s / 1e9 / peak, "traffic": None,
            "bytes_per_launch": float(hbm_bytes), "peak_source": peak_src}
    nvlink = {"bytes_received_per_rank": link_bytes, "gbs": link_bytes / step_s / 1e9,
              "peak": 770.0, "peak_source": "measured peer copy, per direction"}
    if rank == 0:
        line = {
            "metric": "join+agg rows/s", "value": value, "unit": "rows/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int64", "data": "synthetic (seeded generator, inputs on the device)",
            "config": {"workload": w.name + f" x{world} (sharded)",
                       "build_rows": w.n_build * world, "probe_rows": w.n_probe * world,
                       "groups": w.n_groups, "fanout_B": B, "parallelism": f"sharded{world}",
                       "l2": "inputs exceed L2; no flush", "groups_out": groups_out,
                       "matched_probe_rows": matched,
                       "rows_moved_per_step": int(moved)},
            "roofline": roof, "nvlink": nvlink,
            "e2e": e2e, "clocks": clocks, "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)


def run_plain_form(args, w, dev, inputs, keys, sums, counts, our_ms):
    """The reference's own GPU path on the same inputs (its compiled
    partition_sort and join_unique_hash kernels, torch between them, composed
    as its UVM executor does: oracle/plain_form.py), checked equal to ours,
    then timed with CUDA events over a few steps."""
    import torch
    from oracle import plain_form
    if not plain_form.available():
        return {"unavailable": "the reference's kernels are not built (oracle/build_ref.sh)"}
    k, s, c = plain_form.join_aggregate(*inputs, w.scale)
    same = bool(torch.equal(k, keys) and torch.equal(s, sums) and torch.equal(c, counts))
    del k, s, c
    steps = max(1, args.plain_steps)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        plain_form.join_aggregate(*inputs, w.scale)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    torch.cuda.empty_cache()
    return {"value": (w.n_build + w.n_probe) / (ms / 1e3), "unit": "rows/s", "ms_per_step": ms,
            "steps": steps, "identical_results": same, "speedup": ms / our_ms,
            "kind": "the reference's operators/kernels compiled for sm_100a + its torch "
                    "composition restated step for step (uvm/join.py:98-225, "
                    "uvm/aggregate.py:147-212: KeyedAggregate.pass1 per morsel with the "
                    "seeded coefficients, reduce_tick_slice per round)"}


def run_e2e(args, w, plan, dev, dev_inputs, world):
    """The same metric with the inputs in pinned host memory, through
    JoinAggregate.run_stream: every step's columns cross the host link (a
    step's copy overlapping the join of the step before it) and every step's
    groups come back to pinned host memory (device-timed, max over ranks)."""
    import torch
    import torch.distributed as dist
    host = tuple(t.cpu().pin_memory() for t in dev_inputs)
    h2d = sum(t.numel() * t.element_size() for t in host)
    stream = torch.cuda.current_stream(dev)
    for _ in plan.run_stream([host]):   # its device buffers, once
        pass
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    d2h = 0
    for out in plan.run_stream([host] * args.e2e_steps):
        d2h = sum(x.numel() * x.element_size() for x in out)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
    value = job_rate((w.n_build + w.n_probe) * args.e2e_steps, ms, world)
    return {"value": value, "unit": "rows/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": ms / args.e2e_steps,
            "h2d_gbs": h2d / (ms / args.e2e_steps / 1e3) / 1e9,
            "pipeline": "a step's host-to-device copy overlaps the join of the step before it"}


def run_batch(args, world, rank, local_rank):
    """The batching workload at its stated size: all 4,096 join + group-by
    instances (seed 3), in waves of whole instances that fit the device
    (--batch-gb of inputs a wave; each wave's inputs generated on the device
    outside the timed region).  A wave runs as one persistent launch
    replayed from a CUDA graph (timed over --steps replays after --warmup);
    the job's time is the sum of its waves'.  Beside it every wave as
    per-instance launches of the fused path, and the reference's own GPU
    path per instance on the first --plain-instances instances."""
    import torch
    from pageflow_b200 import datagen
    from pageflow_b200.batch import BatchJoinAggregate, Instance
    from pageflow_b200.join_aggregate import JoinAggregate

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    specs = [sp for i, sp in enumerate(datagen.batch_workload(4096, seed=3))
             if i % world == rank]                      # ranks split the job
    budget = args.batch_gb * 1e9
    waves, cur, used = [], [], 0.0
    for sp in specs:
        need = sp.n_build * (12 + 32) + sp.n_probe * 16 + sp.n_groups * 16
        if cur and used + need > budget:
            waves.append(cur)
            cur, used = [], 0.0
        cur.append(sp)
        used += need
    if cur:
        waves.append(cur)
    sampler = ClockSampler(None)
    total_ms, total_rows, pi_ms, same, stats = 0.0, 0, 0.0, True, []
    plain_rows, plain_ms, plain_n = 0, 0.0, 0
    from oracle import plain_form
    want_plain = 0 if args.no_plain_form or not plain_form.available() else \
        (args.plain_instances or 64)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for wave in waves:
        insts = []
        for sp in wave:
            key, grp, fk, val = datagen.gen_batch_instance(sp, dev)
            insts.append(Instance(key, grp, fk, val, 0, sp.n_groups))
        rows = sum(sp.n_build + sp.n_probe for sp in wave)
        b = BatchJoinAggregate(insts, dev)
        g = b.graph()
        for _ in range(args.warmup):
            g.replay()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps):
            g.replay()
        e1.record()
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1) / args.steps
        total_rows += rows
        stats.append(b.read_stats())
        # the same instances, one fused-path launch sequence each
        plans = [JoinAggregate(x.build_key.numel(), x.probe_fk.numel(), 0, x.n_groups, dev,
                               scale=0, autotune=False) for x in insts]

        def per_instance():
            for p, x in zip(plans, insts):
                p.aggregate(x.build_key, x.build_group, x.probe_fk, x.probe_value, None)
        per_instance()
        torch.cuda.synchronize()
        same = same and all(torch.equal(p.sum, b.result(i)[0]) and
                            torch.equal(p.count, b.result(i)[1])
                            for i, p in enumerate(plans[:64]))
        e0.record()
        per_instance()
        e1.record()
        torch.cuda.synchronize()
        pi_ms += e0.elapsed_time(e1)
        del plans
        # the reference's GPU path per instance, on the job's first instances
        k = min(len(insts), want_plain - plain_n)
        if k > 0:
            def plain_run():
                for x in insts[:k]:
                    plain_form.join_aggregate(x.build_key, x.build_group, x.probe_fk,
                                              x.probe_value, torch.zeros_like(x.probe_value), 1)
            plain_run()
            torch.cuda.synchronize()
            e0.record()
            plain_run()
            e1.record()
            torch.cuda.synchronize()
            plain_ms += e0.elapsed_time(e1)
            plain_rows += sum(x.build_key.numel() + x.probe_fk.numel() for x in insts[:k])
            plain_n += k
        del g, b, insts
        torch.cuda.empty_cache()
    clocks = sampler.stop()
    ms = max_over_ranks(total_ms, world, dev)
    all_rows = sum_over_ranks(total_rows, world, dev)
    if rank == 0:
        agg = {k: sum(s_[k] for s_ in stats) for k in stats[0]} if stats else {}
        value = all_rows / (ms / 1e3)
        pi_value = total_rows / (pi_ms / 1e3)
        plain = None
        if plain_n:
            pv = plain_rows / (plain_ms / 1e3)
            plain = {"value": pv, "unit": "rows/s", "instances": plain_n, "ms": plain_ms,
                     "speedup": value / pv if world == 1 else None}
        line = {
            "metric": "join+agg rows/s (batched)", "value": value,
            "unit": "rows/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded, on device)",
            "config": {"workload": "batch: 4096 instances (seed 3), all of them",
                       "instances": len(specs), "waves": len(waves), "rows": total_rows,
                       "wave_budget_gb": args.batch_gb,
                       "skews": sorted({sp.skew for sp in specs})},
            "stats": agg,
            "per_instance_launches": {"value": pi_value, "ms": pi_ms,
                                      "identical_results": same,
                                      "speedup": value / pi_value if world == 1 else None},
            "plain_form_per_instance": plain, "clocks": clocks,
        }
        print(json.dumps(line), flush=True)


def paged_kept_rows(spec) -> int:
    """Rows of the paged table whose date passes the filter, from the date
    column's closed form (date = 8035 + ((r mod 2^20) * 2557) >> 20)."""
    import numpy as np
    cyc = 1 << 20
    d = 8035 + ((np.arange(cyc, dtype=np.int64) * 2557) >> 20)
    ok = (d >= spec.date_lo) & (d < spec.date_hi)
    full, rest = divmod(spec.n_rows, cyc)
    return int(ok.sum()) * full + int(ok[:rest].sum())


def h2d_peak_gbs(dev, nbytes=2 << 30) -> float:
    """A plain pinned host -> device copy's rate on this box (best of 5)."""
    import torch
    src = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    dst = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dst.copy_(src, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, nbytes / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del src, dst
    return best


def run_paged(args, world, rank, local_rank):
    """The paged workload (seed 2): 2.4B rows x 6 columns as PFC1 pages in
    pinned host memory (generated and encoded on the host, untimed); a step
    is one decode -> date filter -> radix partition pass over the whole
    table, the compressed pages crossing the link inside the timed region.
    Reports the effective uncompressed link rate (raw table bytes / s), the
    compressed link rate against a plain pinned copy's, and HBM bytes / s."""
    import numpy as np
    import torch
    import oracle
    from pageflow_b200 import _native, paged

    name = args.workload
    spec = paged.PAGED
    if "/" in name:
        spec = paged.scaled(spec, float(name.split("/", 1)[1]))
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    t0 = time.perf_counter()
    table = paged.PagedTable.generate(spec)
    gen_s = time.perf_counter() - t0
    kept = paged_kept_rows(spec)
    B = args.B or 256
    gpb = 64
    scan = paged.PagedScan(table, "date", spec.date_lo, spec.date_hi, "fk", B=B,
                           groups_per_batch=gpb,
                           capacity_rows=kept + spec.rows_per_page * gpb)
    for _ in range(args.warmup):
        parts = scan.run()
    torch.cuda.synchronize()
    st = parts.read_stats()
    offs = parts.bucket_offsets.cpu().numpy()
    # checks: the kept rows (closed form), the batch totals, and a sample of
    # rows in their buckets (oracle mix64)
    ok_rows = st["rows"] == kept and int(offs[:, B].sum()) == kept and st["bad_pages"] == 0
    k = offs.shape[0] // 2
    lo_r, hi_r = int(offs[k, 0]), int(offs[k, 0] + offs[k, B])
    fk = parts.columns["fk"][lo_r:hi_r].cpu().numpy()
    bk = oracle.bucket(fk, B)
    want = np.repeat(np.arange(B), np.diff(np.append(offs[k, :B], offs[k, 0] + offs[k, B])))
    ok_buckets = bool(np.array_equal(bk, want))

    sampler = ClockSampler(None)
    time.sleep(0.3)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = _native.launch_count()
    _native.profile_begin()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        scan.run()
    e1.record(stream)
    torch.cuda.synchronize()
    prof = _native.profile_end()
    launches = _native.launch_count() - launches0
    clocks = sampler.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world, dev) / args.steps

    # end to end: the same pass plus the bucket offsets and counters read back
    e0.record(stream)
    for _ in range(args.e2e_steps):
        p = scan.run()
        offs_h = p.bucket_offsets.to("cpu", non_blocking=True)
        st_h = p.stats.to("cpu", non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world, dev) / args.e2e_steps
    d2h = offs_h.numel() * 8 + st_h.numel() * 8

    peak, peak_kind = measured_peak()
    link_peak = h2d_peak_gbs(dev)
    comp = table.total_bytes
    raw = table.raw_bytes
    out_bytes = kept * (8 + 8 + 8 + 4 + 4)
    hbm_alg = 2 * comp + out_bytes      # pages land once and are read once; rows written once
    kernels = {n: {"ms_per_step": v[0] / args.steps, "launches_per_step": v[1] / args.steps}
               for n, v in prof.items()}
    scat = prof.get("k_paged_scatter")
    roofline = None
    if scat:
        per_launch_ms = scat[0] / scat[1]
        n_launch_step = scat[1] / args.steps
        # the scatter reads every page of the batch and writes the kept rows
        alg_launch = (comp + out_bytes) / n_launch_step
        ach = alg_launch / (per_launch_ms / 1e3) / 1e9
        roofline = {"bound": "hbm", "kernel": "k_paged_scatter", "achieved": ach, "peak": peak,
                    "unit": "GB/s", "frac": ach / peak, "traffic": None,
                    "bytes_per_launch": alg_launch, "peak_source": peak_kind}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = paged_cpu_baseline(table, spec)
    if rank == 0:
        line = {
            "metric": "paged scan effective link GB/s (uncompressed bytes / s)",
            "value": world * raw / (ms / 1e3) / 1e9, "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int64/int32", "data": "synthetic (seeded generator, PFC1 pages in "
                                            "pinned host memory)",
            "config": {"workload": name, "rows": spec.n_rows, "columns": list(table.names),
                       "rows_per_page": spec.rows_per_page, "groups_per_batch": gpb,
                       "fanout_B": B, "filter": f"{spec.date_lo} <= date < {spec.date_hi}",
                       "kept_rows": kept, "raw_bytes": raw, "compressed_bytes": comp,
                       "ratio": raw / comp, "generate_s": gen_s,
                       "l2": "pages stream from the host: every step is cold"},
            "rows_per_s": world * spec.n_rows / (ms / 1e3),
            "link": {"compressed_gbs": comp / (ms / 1e3) / 1e9, "h2d_copy_peak_gbs": link_peak,
                     "frac": comp / (ms / 1e3) / 1e9 / link_peak},
            "hbm": {"algorithmic_bytes": hbm_alg, "gbs": hbm_alg / (ms / 1e3) / 1e9,
                    "peak": peak, "frac": hbm_alg / (ms / 1e3) / 1e9 / peak},
            "roofline": roofline, "kernels": kernels,
            "checks": {"kept_rows": ok_rows, "buckets_sample": ok_buckets, "stats": st},
            "e2e": {"value": world * raw / (e2e_ms / 1e3) / 1e9, "unit": "GB/s",
                    "h2d_bytes_per_step": comp, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_ms},
            "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)


def paged_cpu_baseline(table, spec, seconds: float = 10.0):
    """The oracle's decode -> filter -> partition on every host thread over
    the table's first row groups (about `seconds` of work): decoded bytes /
    s, uncompressed."""
    import numpy as np
    from concurrent.futures import ThreadPoolExecutor
    import oracle
    threads = oracle.threads()
    pages = table.pages.numpy()
    ends = np.append(table.directory[1:], table.total_bytes)
    nc = len(table.names)
    fc, kc = table.names.index("date"), table.names.index("fk")

    def group(g):
        cols = [oracle.page_decode(pages[table.directory[g * nc + c]:ends[g * nc + c]])
                for c in range(nc)]
        keep = (cols[fc] >= spec.date_lo) & (cols[fc] < spec.date_hi)
        bk = oracle.bucket(cols[kc][keep], 256)
        order = np.argsort(bk, kind="stable")
        return [c[keep][order] for i, c in enumerate(cols) if i != fc]

    done, t0 = 0, time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        while time.perf_counter() - t0 < seconds and done < table.n_groups:
            n = min(threads, table.n_groups - done)
            list(ex.map(group, range(done, done + n)))
            done += n
    el = time.perf_counter() - t0
    rows = min(table.n_rows, done * table.rows_per_page)
    raw = rows * sum(table.esizes)
    return {"value": raw / el / 1e9, "unit": "GB/s", "cores": threads, "kind": "port",
            "sample": f"the first {done} row groups ({rows} rows), {el:.1f} s"}


def _plain_request(dims, fact, r):
    """One serving request the reference's way: the range mask, mask
    compaction, then the plain-form join + group-by on the GPU."""
    import torch
    from oracle import plain_form
    s = slice(r.row0, r.row0 + r.n_rows)
    d = fact.date[s]
    keep = (d >= r.date_lo) & (d < r.date_hi)
    fk = fact.fk[s][keep]
    val = fact.value[s][keep]
    if fk.numel() == 0:
        e = torch.empty(0, dtype=torch.int64, device=fk.device)
        return e, e, e
    return plain_form.join_aggregate(dims.keys[r.dim], dims.groups[r.dim], fk, val,
                                     torch.zeros_like(val), 1)


def run_serve(args, world, rank, local_rank):
    """The serving workload (seed 4): 8 resident dimensions (1e5 to 2e8
    keys) with persistent hash tables, a resident 1e9-row fact pool, and a
    trace of requests (probe rows log-uniform in [1e5, 1e9], selectivity
    uniform in [1%, 50%]) replayed as Poisson arrivals at each rate of the
    sweep, admitted by a 150 GB HBM budget and batched into persistent
    launches.  Beside it the reference's plain form per request (service
    times measured one by one, queued FIFO at the same arrivals)."""
    import numpy as np
    import torch
    from pageflow_b200 import _native, serve

    name = args.workload
    spec = serve.SERVE if "/" not in name else serve.scaled(serve.SERVE,
                                                            float(name.split("/", 1)[1]))
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    t0 = time.perf_counter()
    dims = serve.Dimensions(spec, dev)
    fact = serve.FactPool(spec, dev)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    n = args.serve_requests
    trace = serve.make_requests(spec, n, seed=spec.seed + 1000 * rank)
    rates = [float(x) for x in args.serve_rates.split(",")]
    srv = serve.Server(dims, fact, spec.budget_bytes, dev, iter_rows=args.serve_iter_rows)

    def fresh(rate):
        out = []
        arr = serve.poisson_arrivals(n, rate, seed=spec.seed) if rate > 0 else np.zeros(n)
        for r, a in zip(trace, arr):
            out.append(serve.Request(r.id, r.dim, r.row0, r.n_rows, r.date_lo, r.date_hi,
                                     float(a)))
        return out

    # warm-up and the results every later run is checked against: a burst
    for _ in range(max(1, args.warmup)):
        burst = fresh(0)
        srv.run(burst, keep_results=True)
    ours = {r.id: r.result for r in burst}
    sampler = ClockSampler(None)
    launches0 = _native.launch_count()
    sweep = []
    for rate in rates:
        reqs = fresh(rate)
        run = srv.run(reqs, keep_results=False)
        lat = run.latencies() * 1e3
        span = max(r.t_done for r in reqs) - min(r.arrival for r in reqs)
        sweep.append({"rate": rate, "p50_ms": float(np.percentile(lat, 50)),
                      "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
                      "completed_per_s": n / span, "rows_per_s": run.rows / span,
                      "launches": run.launches, "max_admitted": run.max_admitted,
                      "wall_s": run.wall_s})
    launches = _native.launch_count() - launches0
    clocks = sampler.stop()
    rows_total = sum(r.n_rows for r in trace)
    del srv
    torch.cuda.empty_cache()

    # the plain form, one request at a time, each checked against ours
    plain = None
    from oracle import plain_form
    if plain_form.available() and not args.no_plain_form:
        svc = np.zeros(n)
        same = True
        for r in trace:
            torch.cuda.synchronize()
            a = time.perf_counter()
            k, s, c = _plain_request(dims, fact, r)
            torch.cuda.synchronize()
            svc[r.id] = time.perf_counter() - a
            mine = ours[r.id]
            same &= bool(np.array_equal(k.cpu().numpy(), mine[0]) and
                         np.array_equal(s.cpu().numpy(), mine[1]) and
                         np.array_equal(c.cpu().numpy(), mine[2]))
            del k, s, c
        for entry in sweep:
            lat = serve.lindley(serve.poisson_arrivals(n, entry["rate"], seed=spec.seed),
                                svc[[r.id for r in trace]]) * 1e3
            entry["plain_p50_ms"] = float(np.percentile(lat, 50))
            entry["plain_p99_ms"] = float(np.percentile(lat, 99))
        plain = {"rows_per_s": rows_total / svc.sum(), "service_ms_mean": svc.mean() * 1e3,
                 "identical_results": same,
                 "kind": "mask + compaction (torch) + the reference's compiled partition_sort / "
                         "join_unique_hash + its torch group-by, one request at a time; "
                         "latency = FIFO queue over the measured service times"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = serve_cpu_baseline(spec, dims, fact, trace)
    top = sweep[-1]
    job_rows_per_s = sum_over_ranks(top["rows_per_s"], world, dev)
    # the knee: the highest rate still served as offered (completions keep up
    # with the trace's realised arrival rate) with p99 within 10x of the
    # lowest rate's
    knee = None
    base_p99 = sweep[0]["p99_ms"]
    for e in sweep:
        arr = serve.poisson_arrivals(n, e["rate"], seed=spec.seed)
        offered = (n - 1) / (arr[-1] - arr[0])
        e["offered_per_s"] = offered
        if e["completed_per_s"] >= 0.95 * offered and e["p99_ms"] <= 10 * base_p99:
            knee = e["rate"]
    res_bytes = float(np.mean([24 * ours[i][0].shape[0] for i in ours]))
    if rank == 0:
        line = {
            "metric": "serving rows/s at the highest offered rate; p50/p99 latency per rate",
            "value": job_rows_per_s, "unit": "rows/s", "n_gpus": world,
            "steps": n, "warmup": args.warmup, "ms_per_step": 1e3 / top["completed_per_s"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int64", "data": "synthetic (seeded generator, resident on the device)",
            "config": {"workload": name, "requests": n, "rates": rates,
                       "dims_keys": list(spec.dim_keys), "dims_groups": list(spec.dim_groups),
                       "fact_rows": spec.fact_rows, "budget_gb": spec.budget_bytes / 1e9,
                       "iter_rows": args.serve_iter_rows, "trace_rows": rows_total,
                       "setup_s": setup_s,
                       "l2": "requests scan slices of a 20 GB fact pool, far above L2"},
            "sweep": sweep, "knee_rate": knee, "plain_form": plain,
            "e2e": {"value": job_rows_per_s, "unit": "rows/s",
                    "h2d_bytes_per_step": 128, "d2h_bytes_per_step": res_bytes,
                    "note": "a step is one request: its descriptor in, its groups back"},
            "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)


def serve_cpu_baseline(spec, dims, fact, trace, seconds: float = 10.0):
    """The oracle's filter + join + group-by on every host thread over the
    trace's requests against dimensions of at most 3M keys (their rows
    copied to the host), for about `seconds`: probe rows / s."""
    import oracle
    oracle.build()
    cpu_dims = {}
    rows = 0
    t_run = 0.0
    done = 0
    for r in trace:
        if spec.dim_keys[r.dim] > 3_000_000 or r.n_rows > 20_000_000:
            continue
        if r.dim not in cpu_dims:
            cpu_dims[r.dim] = (dims.keys[r.dim].cpu().numpy(), dims.groups[r.dim].cpu().numpy())
        s = slice(r.row0, r.row0 + r.n_rows)
        fk, d, v = fact.fk[s].cpu().numpy(), fact.date[s].cpu().numpy(), fact.value[s].cpu().numpy()
        k, g = cpu_dims[r.dim]
        a = time.perf_counter()
        oracle.serve_request(k, g, spec.dim_groups[r.dim], fk, d, v, r.date_lo, r.date_hi)
        t_run += time.perf_counter() - a
        rows += r.n_rows
        done += 1
        if t_run >= seconds:
            break
    if not done:
        return None
    return {"value": rows / t_run, "unit": "rows/s", "cores": oracle.threads(), "kind": "port",
            "sample": f"{done} requests of the trace on dimensions of <= 3M keys, "
                      f"{rows} probe rows, {t_run:.1f} s"}


def drop_in_vs_reference(dev, timed, peak):
    """The drop-in kernels against the reference's own CUDA kernels (its
    operators/kernels/*.cu built from source for sm_100a), on the same
    inputs, outputs checked equal: partition_sort of 50M rows (int64 key,
    int64 and int32 payloads) into 256 padded buckets, and join_unique_hash
    of 100M probe rows against 25M unique build keys (90% matching)."""
    import torch
    from oracle import plain_form
    from pageflow_b200 import tqpkernels
    if not plain_form.available():
        return {"drop_in_vs_reference": "unavailable: the reference's kernels are not built"}
    ref = plain_form.kernels()
    g = torch.Generator(device=dev).manual_seed(11)
    out = {}
    n, B = 50_000_000, 256
    cols = [torch.randint(-(1 << 40), 1 << 40, (n,), device=dev, generator=g),
            torch.randint(-(1 << 40), 1 << 40, (n,), device=dev, generator=g),
            torch.randint(-(1 << 30), 1 << 30, (n,), device=dev, generator=g, dtype=torch.int32)]
    h1 = torch.zeros(B + 5, dtype=torch.int64, pin_memory=True)
    h2 = torch.zeros(B + 5, dtype=torch.int64, pin_memory=True)
    comp = [0, 0, 0]
    a = tqpkernels.partition_sort(cols, comp, 0, None, n, 0, B, False, h1)
    b = ref.partition_sort(cols, comp, 0, None, n, 0, B, False, h2)
    torch.cuda.synchronize()
    counts = h1[:B].tolist()

    def real_rows(t):
        # each bucket starts on a whole 512-byte unit of the column; padding
        # rows are never written
        rb = t.element_size() * (t.shape[1] if t.dim() == 2 else 1)
        unit = 512 // math.gcd(rb, 512)
        m = torch.zeros(t.shape[0], dtype=torch.bool, device=t.device)
        at = 0
        for c in counts:
            m[at:at + c] = True
            at += -(-c // unit) * unit
        return m
    same = h1[:B + 4].tolist() == h2[:B + 4].tolist() and len(a) == len(b) and all(
        torch.equal(x[real_rows(x)], y[real_rows(y)]) for x, y in zip(a, b))
    del a, b
    ms = timed(lambda: tqpkernels.partition_sort(cols, comp, 0, None, n, 0, B, False, h1))
    ms_ref = timed(lambda: ref.partition_sort(cols, comp, 0, None, n, 0, B, False, h2))
    # the key read by the count, the columns (key included) read and written
    # by the scatter, the int64 gidx written
    byts = n * (8 + 20 + 20 + 8)
    out["partition_sort_50M_B256"] = {"ms": ms, "gbs": byts / ms / 1e6,
                                      "frac": byts / ms / 1e6 / peak, "reference_ms": ms_ref,
                                      "speedup": ms_ref / ms, "identical": same}
    del cols
    nb, np_ = 25_000_000, 100_000_000
    bk = torch.randperm(nb, device=dev, generator=g).to(torch.int64) * 3 + 1
    pick = torch.randint(0, nb, (np_,), device=dev, generator=g)
    pk = bk[pick]
    miss = torch.rand(np_, device=dev, generator=g) < 0.1
    pk = torch.where(miss, pk + 1, pk)
    h1, h2 = torch.zeros(2, dtype=torch.int64, pin_memory=True), torch.zeros(
        2, dtype=torch.int64, pin_memory=True)
    a = tqpkernels.join_unique_hash([bk], [pk], h1)
    b = ref.join_unique_hash([bk], [pk], h2)
    torch.cuda.synchronize()
    m = int(h1[0])
    same = m == int(h2[0]) and all(torch.equal(x[:m], y[:m]) for x, y in zip(a, b))
    del a, b
    ms = timed(lambda: tqpkernels.join_unique_hash([bk], [pk], h1))
    ms_ref = timed(lambda: ref.join_unique_hash([bk], [pk], h2))
    byts = nb * 8 + np_ * 8 + m * 16
    out["join_unique_hash_25M_x_100M"] = {"ms": ms, "gbs": byts / ms / 1e6,
                                          "frac": byts / ms / 1e6 / peak, "reference_ms": ms_ref,
                                          "speedup": ms_ref / ms, "identical": same}
    return out


def run_kernels(args, world, rank, local_rank):
    """The operator primitives beside the fused path, each timed with CUDA
    events (median of `steps` runs after `warmup`) on inputs far above L2,
    against the reference's plain torch form of the same operation, results
    checked equal: the join tail's gather (two int64 columns at 100M random
    indexes), the radix sort (100M int64 keys over 40 bits), reduce_tick_slice
    (100M rows, 1M keys, two int64 sums), the merge of two 50M-key runs, and
    the keyed pass 1's grouping hash (100M rows, int64 + int32 keys)."""
    import torch
    from pageflow_b200 import gather as G, keyed_aggregate as KA, sorted_run_merge as SRM

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    peak, peak_kind = measured_peak()
    g = torch.Generator(device=dev).manual_seed(7)
    n = 100_000_000

    def timed(fn):
        for _ in range(max(1, args.warmup)):
            fn()
        ts = []
        for _ in range(max(1, args.steps)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    out = {}
    # gather
    a = torch.randint(-(1 << 40), 1 << 40, (n,), device=dev, generator=g)
    b = torch.randint(-(1 << 40), 1 << 40, (n,), device=dev, generator=g)
    idx = torch.randint(0, n, (n,), device=dev, generator=g)
    ours = G.index_select_many([a, b], idx)
    same = all(torch.equal(x, torch.index_select(y, 0, idx)) for x, y in zip(ours, [a, b]))
    ms = timed(lambda: G.index_select_many([a, b], idx))
    ms_ref = timed(lambda: [torch.index_select(a, 0, idx), torch.index_select(b, 0, idx)])
    byts = n * (8 + 2 * 16)
    out["gather_2x_int64"] = {"ms": ms, "gbs": byts / ms / 1e6, "frac": byts / ms / 1e6 / peak,
                              "torch_ms": ms_ref, "identical": same}
    del ours
    # radix sort
    k = torch.randint(0, 1 << 40, (n,), device=dev, generator=g)
    ko, vo = SRM.sort_pairs(k)
    rs, ri = torch.sort(k, stable=True)
    same = bool(torch.equal(ko, rs) and torch.equal(vo, ri))
    ms = timed(lambda: SRM.sort_pairs(k))
    ms_ref = timed(lambda: torch.sort(k, stable=True))
    byts = n * 5 * 32  # 5 passes of 40 bits: 16 B read + 16 B written a key
    out["radix_sort_40bit"] = {"ms": ms, "keys_per_s": n / ms * 1e3, "gbs": byts / ms / 1e6,
                               "frac": byts / ms / 1e6 / peak, "torch_ms": ms_ref,
                               "identical": same}
    del ko, vo, rs, ri
    # reduce_tick_slice
    keys = torch.randint(0, 1 << 20, (n,), device=dev, generator=g)
    v1 = torch.randint(-10**6, 10**6, (n,), device=dev, generator=g)
    v2 = torch.randint(-10**6, 10**6, (n,), device=dev, generator=g)
    u, (s1, s2) = SRM.reduce_tick_slice(keys, [v1, v2], ["sum", "sum"])

    def torch_reduce():
        uu, inv = torch.unique(keys, return_inverse=True)
        r1 = torch.zeros(uu.numel(), dtype=torch.int64, device=dev)
        r1.scatter_reduce_(0, inv, v1, reduce="sum", include_self=False)
        r2 = torch.zeros(uu.numel(), dtype=torch.int64, device=dev)
        r2.scatter_reduce_(0, inv, v2, reduce="sum", include_self=False)
        return uu, r1, r2
    tu, t1, t2 = torch_reduce()
    same = bool(torch.equal(u, tu) and torch.equal(s1, t1) and torch.equal(s2, t2))
    ms = timed(lambda: SRM.reduce_tick_slice(keys, [v1, v2], ["sum", "sum"]))
    ms_ref = timed(torch_reduce)
    out["reduce_tick_slice_1M_keys"] = {"ms": ms, "rows_per_s": n / ms * 1e3,
                                        "torch_ms": ms_ref, "identical": same}
    del u, s1, s2, tu, t1, t2
    # merge of two unique runs
    ra = torch.unique(torch.randint(0, 1 << 34, (n // 2,), device=dev, generator=g))
    rb = torch.unique(torch.randint(0, 1 << 34, (n // 2,), device=dev, generator=g))
    va, vb = torch.ones_like(ra), torch.ones_like(rb)
    cap = ra.numel() + rb.numel()

    def ours_merge():
        kb = torch.empty(cap, dtype=torch.int64, device=dev)
        vv = torch.empty(cap, dtype=torch.int64, device=dev)
        kb[:ra.numel()], vv[:ra.numel()] = ra, va
        m = SRM.merge_sorted_unique_runs_inplace(kb, [vv], ra.numel(), rb, [vb], ["sum"])
        return kb[:m], vv[:m]
    mk, mv = ours_merge()
    uu, inv = torch.unique(torch.cat([ra, rb]), return_inverse=True)
    same = bool(torch.equal(mk, uu) and torch.equal(mv, torch.bincount(inv)))
    ms = timed(ours_merge)
    out["merge_runs_2x50M"] = {"ms": ms, "keys_per_s": cap / ms * 1e3, "identical": same}
    del mk, mv, uu, inv
    # grouping hash
    k1 = torch.randint(-(1 << 40), 1 << 40, (n,), device=dev, generator=g)
    k2 = torch.randint(0, 1 << 30, (n,), device=dev, generator=g, dtype=torch.int32)
    keys2 = [k1.unsqueeze(1), k2.unsqueeze(1)]
    coeffs = KA.make_key_coeffs(keys2, dev)
    h = KA.group_hash(keys2, coeffs)

    def torch_hash():
        return (k1 * coeffs[0][0]) + (k2.to(torch.int64) & 0xFFFFFFFF) * coeffs[1][0]
    same = bool(torch.equal(h, torch_hash()))
    ms = timed(lambda: KA.group_hash(keys2, coeffs))
    ms_ref = timed(torch_hash)
    byts = n * (8 + 4 + 8)
    out["group_hash_int64_int32"] = {"ms": ms, "gbs": byts / ms / 1e6,
                                     "frac": byts / ms / 1e6 / peak, "torch_ms": ms_ref,
                                     "identical": same}
    del h, k1, k2, keys2
    out.update(drop_in_vs_reference(dev, timed, peak))
    if rank == 0:
        line = {"metric": "operator primitives: ms per call (median) and GB/s of algorithmic bytes",
                "value": out["gather_2x_int64"]["gbs"], "unit": "GB/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": out["gather_2x_int64"]["ms"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "int64",
                "data": "synthetic (seeded, on the device, far above L2)",
                "config": {"workload": "kernels", "rows": n, "peak_gbs": peak,
                           "peak_source": peak_kind},
                "kernels": out}
        print(json.dumps(line), flush=True)


def main(argv=None) -> int:
    args = parse_args(argv)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    mode = args.workload.split("/", 1)[0]
    if args.impl == "reference":
        if mode in ("serve", "paged", "batch", "kernels"):
            if rank == 0:
                why = {"serve": "the serve workload's reference arm is its plain form per "
                                "request, reported as plain_form of --workload serve",
                       "paged": "the paged workload's reference arm is the oracle decoder, "
                                "reported as cpu_baseline of --workload paged",
                       "batch": "the batch workload's reference arm is the plain form per "
                                "instance, reported as plain_form_per_instance of --workload "
                                "batch",
                       "kernels": "the primitives' reference arm is their torch plain form, "
                                  "reported as torch_ms of --workload kernels"}[mode]
                print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
            return 0
        run_reference(args, workload(args.workload), world, rank)
        return 0
    run = {"batch": run_batch, "serve": run_serve, "paged": run_paged,
           "kernels": run_kernels}.get(mode)
    w = None if run else workload(args.workload)
    sharded = not run and (args.parallelism == "sharded" or
                           (args.parallelism is None and world > 1))
    if world > 1 or sharded:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        if world == 1:   # a one-rank group of this process (no launcher)
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            os.environ.setdefault("MASTER_PORT", "29571")
            os.environ.setdefault("RANK", "0")
            os.environ.setdefault("WORLD_SIZE", "1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        if run:
            run(args, world, rank, local_rank)
        elif sharded:
            run_sharded(args, w, world, rank, local_rank)
        else:
            run_ours(args, w, world, rank, local_rank)
    finally:
        if world > 1 or sharded:
            import torch.distributed as dist
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
