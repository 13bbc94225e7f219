#!/usr/bin/env python
"""Benchmark of the del3d Delaunay::build hot path on B200.

Workload: one plain single-set build per step of 1e7 points i.i.d. uniform in
[0,1)^3 (std::mt19937, u01 = word * 2^-32; seed 6 + rank), float64.  With
N > 1 GPUs each rank builds its own set (replicas, weak scaling); there is no
exchange step in a Delaunay build of independent sets.

One JSON line (rank 0):
  value      points/s of the whole job, inputs resident in HBM, device-timed
             with CUDA events on the build's stream (max over ranks);
  e2e        the same metric through the host C ABI d3g_build (pinned host
             input copied in, finite_cells + all_cells + incident_cells copied
             back every step), which is what a del3d caller gets;
  roofline   the dominant insertion kernel: algorithmic bytes it must touch
             (live counts) / its event-timed duration, against measured HBM;
  cpu_baseline  the reference del3d compiled from source, single thread, on a
             1e6-point sample of the same distribution (rank 0, N = 1).

`--impl reference` times the reference's own CPU build instead (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "points/sec batched vs plain GPU at bit-exact tet sets; p50/p99 latency"
N_POINTS = 10_000_000
SEED = 6
CPU_SAMPLE = 1_000_000
HBM_FALLBACK_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_POINTS)
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": HBM_FALLBACK_GBS}, "fallback"


def workload(n):
    return {"workload": f"plain single-set Delaunay build, {n:.0e} points uniform in [0,1)^3 "
                        f"(mt19937 seed {SEED}+rank), float64",
            "points_per_set": n, "sets_per_gpu_per_step": 1, "parallelism": "replicas",
            "l2": "inputs larger than L2 (24 B/point points, ~57 B/tet tables)"}


class Clocks:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id: str):
        self.p = None
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", device_id], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.p.kill()
            out, _ = self.p.communicate()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for name, flag in zip(names, f[3:7]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def gpu_id(torch, dev):
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return str(dev)


def count_launches(torch, fn):
    """Kernels one call of fn launches (CUDA activity from the profiler)."""
    try:
        from torch.profiler import ProfilerActivity, profile

        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            fn()
            torch.cuda.synchronize()
        return sum(1 for e in prof.events() if e.device_type.name == "CUDA" and
                   "memcpy" not in e.name.lower() and "memset" not in e.name.lower())
    except Exception:
        return None


def cpu_baseline_leg():
    import oracle
    import del3d_b200 as d3

    if not oracle.ref_available():
        return None
    pts = d3.gen_uniform(CPU_SAMPLE, SEED)
    import ctypes
    import numpy as np

    nc = ctypes.c_int64(0)
    t = oracle.ref().ref_build_time(pts.ctypes.data, pts.shape[0], ctypes.byref(nc))
    return {"value": CPU_SAMPLE / t, "unit": "points/s", "cores": 1, "kind": "reference",
            "sample": f"one reference Delaunay::build of {CPU_SAMPLE:.0e} points of the same "
                      f"distribution (seed {SEED}), {t:.2f} s, single-threaded as the reference is"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import ctypes

    import del3d_b200 as d3
    import oracle

    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
        return 0
    pts = d3.gen_uniform(CPU_SAMPLE, SEED)
    nc = ctypes.c_int64(0)
    times = []
    for step in range(args.warmup + args.steps):
        t = oracle.ref().ref_build_time(pts.ctypes.data, pts.shape[0], ctypes.byref(nc))
        if step >= args.warmup:
            times.append(t)
    value = CPU_SAMPLE * len(times) / sum(times)
    cfg = workload(args.n)
    cfg["reference_sample"] = f"{CPU_SAMPLE:.0e} points per step (a bounded sample of the workload)"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "points/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfg,
            "cpu_baseline": {"value": value, "unit": "points/s", "cores": 1, "kind": "reference",
                             "sample": f"{CPU_SAMPLE:.0e} uniform points per step, one thread "
                                       "(the reference build is single-threaded)"},
            "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args):
    import numpy as np
    import torch

    import del3d_b200 as d3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n = args.n
    host = d3.gen_uniform(n, SEED + rank)
    x = torch.from_numpy(host).to(dev)
    out = torch.empty((8 * n + 64, 4), dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    handle = stream.cuda_stream

    def step(timing=False, stats=None):
        return d3.build_device(x, out=out, stream=handle, chunk=args.chunk, timing=timing,
                               stats=stats)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()

    # ---- timed region: device-resident inputs ----
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(gpu_id(torch, dev)) if rank == 0 else None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ncells = 0
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            cells, nv = step()
            ncells = cells.shape[0]
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else None
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1) / args.steps
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * n / (ms_max / 1000.0)

    # ---- instrumented (untimed) step: per-kernel times and live counts ----
    stats = {}
    with torch.cuda.stream(stream):
        step(timing=True, stats=stats)
    torch.cuda.synchronize()
    launches_per_step = count_launches(torch, lambda: step())

    # ---- end to end through the host C ABI ----
    pinned = torch.from_numpy(host).pin_memory()
    pin_np = pinned.numpy()
    d = d3.Delaunay()
    d.build(pin_np)   # warm
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        d.build(pin_np)
    t_e2e = (time.perf_counter() - t0) / args.steps
    te = torch.tensor([t_e2e], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * n / float(te.item())
    off, inc = d.incident_csr()
    d2h = 16 * (d.finite_cells().shape[0] + d.all_cells().shape[0]) + 8 * off.shape[0] + 4 * inc.shape[0]

    if rank == 0:
        peaks, peak_kind = measured_peaks()
        hbm = float(peaks.get("hbm_gbs", HBM_FALLBACK_GBS))
        # Dominant insertion kernel and its algorithmic bytes: every insertion
        # reads the vertex record (16 B) and claim word (8 B) of each region and
        # ring tet, the neighbour record (16 B) of each region tet, and writes
        # one tet (32 B) per boundary facet.
        kern = {"k_cavity": stats.get("ms_cavity", 0.0), "k_check": stats.get("ms_check", 0.0),
                "k_restar": stats.get("ms_restar", 0.0)}
        dom = max(kern, key=kern.get)
        C, F = stats.get("region_tets", 0), stats.get("boundary_facets", 0)
        launches = max(1, stats.get("launches_cavity", 1))
        bytes_kernel = {"k_cavity": 24 * (C + F) + 16 * C, "k_check": 8 * (C + F) + 16 * F,
                        "k_restar": 32 * C + 32 * F + 40 * F}[dom]
        achieved = (bytes_kernel / launches) / (kern[dom] / launches / 1000.0) / 1e9 if kern[dom] else 0.0
        traffic = None
        prof = os.path.join(ROOT, "profiles", "traffic_per_attempt.json")
        if os.path.exists(prof):
            try:
                with open(prof) as f:
                    per_attempt = json.load(f).get(dom)
                if per_attempt:
                    traffic = per_attempt * stats.get("attempts", 0) / launches
            except (OSError, ValueError):
                traffic = None
        line = {
            "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload(n),
            "e2e": {"value": e2e_value, "unit": "points/s", "h2d_bytes_per_step": 24 * n,
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                         "traffic": traffic,
                         "build_gbs": 132.0 * n / (ms_max / 1000.0) / 1e9,
                         "build_frac": 132.0 * n / (ms_max / 1000.0) / 1e9 / hbm},
            "gpu_launches": (launches_per_step * args.steps) if launches_per_step else None,
            "clocks": clk,
            "build_stats": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in stats.items()},
            "cells": ncells,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_leg()
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
