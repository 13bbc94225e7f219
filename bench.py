#!/usr/bin/env python
"""Benchmark of the del3d Delaunay::build hot path on B200.

Workload (one step): the mixed batched workload - 4096 independent point sets,
sizes log-uniform in [32, 65536], each drawn with equal probability from the
uniform cube [0,1)^3, 8 Gaussian clusters (sigma 0.02), the integer lattice or
the unit sphere quantised to a 2^-10 grid (duplicates removed), float64, per-set
seeds (del3d_b200.mixed_workload).  All sets go to the GPU in one batched build
(d3g_build_batch_device); every set's tet set is the reference's.  With N > 1
GPUs each rank builds its own 4096 sets (weak scaling, no exchange step: sets
are independent); `--scaling strong` splits one 4096-set workload among the
ranks by estimated cost instead (del3d_b200.partition_sets).  The whole-job
rate is every rank's points over the slowest rank's time.

One JSON line (rank 0):
  value       points/s of the whole job, inputs resident in HBM, device-timed
              with CUDA events on the build's stream (max over ranks);
  e2e         the same metric through the host C ABI d3g_build_batch: pinned
              host input copied in, every set's finite cells copied back, each
              step;
  plain       the plain one-set-per-call GPU path (d3g_build_device) on a
              1-in-8 sample of the same sets: points/s and per-set latency
              p50/p99, and batched/plain;
  latency     per-set latency of both forms (a batched set completes with its
              batch);
  roofline    the dominant insertion kernel: algorithmic bytes it must touch
              (live counts) / its event-timed duration, against measured HBM;
  cpu_baseline  the reference del3d compiled from source on a 1-in-16 sample of
              the sets, one set per host thread.
  parity      the parity check: the timed build's cells of every 64th set against
              the reference's build of the same set in canonical order; the run
              exits 1 when they differ.
  plain_1e7   the plain path on 1e7 uniform points and the reference's
              single-threaded build rate on 1e6 of them.
  serving     the request server (d3g_server_*, continuous batching, admission
              by device-memory budget) under Poisson arrivals swept over
              several rates, request sizes log-uniform in [100, 1e6] points of
              the same four distributions: points/s, requests/s and p50/p99
              latency per rate.

Before the warm-up (not timed), d3g_autotune_device times the candidate speed
settings (schedule, worker density, lanes) on every 8th set and makes the fastest
the device default; the line reports the choice under "tuning".

`--impl reference` times the reference's own CPU build on the same sample
(rank 0 only; all host threads, one set per thread).

`--workload readers` (host only, no GPU): every 16th set of the batched workload
written to files in turn as "x y z" text, binary PLY, OBJ and OFF; a step reads
them all with d3g_load_point_sets (all host threads) into the back-to-back layout
of a batched build; cpu_baseline is the reference viewer's reader
(viewer/mesh_io.cpp, compiled from source) on the same files with the same
threads, and the line says whether the points read are the reference's.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time
from concurrent.futures import ThreadPoolExecutor

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "points/sec batched vs plain GPU at bit-exact tet sets; p50/p99 latency"
N_SETS = 4096
LO, HI = 32, 65536
PLAIN_EVERY = 8
CPU_EVERY = 16
PLAIN_N = 10_000_000
PLAIN_SEED = 6
REF_PLAIN_SAMPLE = 1_000_000
HBM_FALLBACK_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched",
                    choices=["batched", "plain", "c3", "predicates", "sort", "readers"],
                    help="batched: the headline line; plain: one single-set build per step "
                         "(--n uniform points); c3: the four plain single-set configurations "
                         "(1e6 uniform, the 100^3 lattice, 1e6 quantised sphere, 1e7 uniform), "
                         "each timed and compared with the reference's build; predicates / sort: "
                         "the predicate and "
                         "spatial-sort microbenchmarks, one line each; readers: the host "
                         "input readers on files of a sample of the batched sets (no GPU)")
    ap.add_argument("--n", type=int, default=PLAIN_N, help="points of the plain workload")
    ap.add_argument("--queries", type=int, default=0,
                    help="predicates workload: queries of each kind (default 1e8); a smaller count "
                         "serves one-kernel profiler captures")
    ap.add_argument("--dist", default="uniform", choices=["uniform", "clusters", "lattice", "sphere"],
                    help="distribution of the plain workload")
    ap.add_argument("--schedule", type=int, default=0,
                    help="0: asynchronous insertion (default); 1: lockstep rounds only")
    ap.add_argument("--timing", action="store_true",
                    help="plain workload: launch each round's kernels separately with event "
                         "timing (the form the ncu launch list captures)")
    ap.add_argument("--sets", type=int, default=N_SETS)
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"],
                    help="N > 1 GPUs: weak - every rank builds its own --sets sets (the default); "
                         "strong - the ranks share one --sets workload, split by estimated cost "
                         "(del3d_b200.partition_sets)")
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--parity-every", type=int, default=0,
                    help="parity leg: check the cells of every k-th set (default 64; 1 checks every set)")
    ap.add_argument("--profile-run", action="store_true",
                    help="warm-up and timed steps only (no other legs): the command profiled by ncu")
    return ap.parse_args()


def job_rate(dist, device, units, seconds):
    """Whole-job rate over the ranks: the units all ranks processed (their sets
    differ in size) over the slowest rank's time.  Every rank calls it at the
    same point, in the same order (two collectives).  Returns (rate, max
    seconds, total units)."""
    import torch

    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(u, op=dist.ReduceOp.SUM)
    t_max, total = float(t.item()), float(u.item())
    return total / t_max, t_max, total


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": HBM_FALLBACK_GBS}, "fallback"


def workload_sets(n_sets, rank, gen=None):
    """The sets of rank `rank`.  `gen` is the module whose generators make them:
    del3d_b200 for our arm, the oracle's copy of the same generators for the
    reference arm (which must not load the product library)."""
    if gen is None:
        import del3d_b200 as gen

    return gen.mixed_workload(n_sets, LO, HI, seed=2024 + rank, first_seed=1000 + n_sets * rank)


def rank_sets(n_sets, rank, world, scaling):
    """The sets rank `rank` builds: its own n_sets sets (weak scaling), or its
    share of one n_sets workload split by estimated cost (strong scaling; every
    rank generates the same workload and keeps its part, so nothing is sent)."""
    if scaling == "weak" or world == 1:
        return workload_sets(n_sets, rank)
    import del3d_b200 as d3

    sets = workload_sets(n_sets, 0)
    part = d3.partition_sets([a.shape[0] for a in sets], world)[rank]
    return [sets[k] for k in part]


def config(n_sets, n_points):
    return {"workload": f"batched Delaunay builds: {n_sets} point sets, sizes log-uniform in "
                        f"[{LO}, {HI}], uniform cube / 8-cluster Gaussian (sigma 0.02) / integer "
                        f"lattice / quantised unit sphere (2^-10 grid, deduplicated), float64, "
                        f"per-set seeds",
            "sets_per_gpu_per_step": n_sets, "points_per_gpu_per_step": n_points,
            "parallelism": "independent sets per GPU (replicas)",
            "l2": "inputs larger than L2 (24 B/point, ~0.85 GB of points per step)"}


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


def pct(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = min(len(xs) - 1, max(0, int(round(q / 100.0 * (len(xs) - 1)))))
    return xs[k]


# ---- the reference's CPU build (oracle/_ref: the reference compiled from its own sources) ----


def reference_build_sets(sets, threads):
    """Builds every set with the reference (one set per host thread at a time).
    Returns (wall seconds, sum of per-set build seconds, points)."""
    import oracle

    lib = oracle.ref()

    def one(a):
        nc = ctypes.c_int64(0)
        return lib.ref_build_time(a.ctypes.data, a.shape[0], ctypes.byref(nc))

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        per_set = list(ex.map(one, sets))
    wall = time.perf_counter() - t0
    return wall, sum(per_set), sum(a.shape[0] for a in sets)


def host_threads():
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return max(1, os.cpu_count() or 1)


def cpu_sample(sets):
    # Largest first so the thread pool does not end on one long set.
    sample = sets[::CPU_EVERY]
    return sorted(sample, key=lambda a: -a.shape[0])


def cpu_baseline_leg(sets):
    import oracle

    if not oracle.ref_available():
        return None
    sample = cpu_sample(sets)
    threads = host_threads()
    wall, cpu_s, pts = reference_build_sets(sample, threads)
    return {"value": pts / wall, "unit": "points/s", "cores": threads, "kind": "reference",
            "sample": f"every {CPU_EVERY}th set of the workload ({len(sample)} sets, {pts} points), "
                      f"one set per thread on {threads} host threads; {wall:.2f} s wall, "
                      f"{cpu_s:.2f} s of single-thread build time "
                      f"({pts / cpu_s:.0f} points/s per thread)"}


PARITY_EVERY = 64


def parity_leg(sets, gpu_cells, every=PARITY_EVERY):
    """Parity: the cells the timed batched build gave every PARITY_EVERY-th
    set (`gpu_cells`: set index -> host array) against the reference's build of
    that set (oracle/_ref), put in the same canonical order; one set per host
    thread.  None when the reference library is absent."""
    import numpy as np

    import oracle

    if not oracle.ref_available() or not gpu_cells:
        return None

    def one(k):
        want = oracle.canonical_cells(oracle.ref_build(sets[k])["cells"])
        return bool(np.array_equal(gpu_cells[k], want))

    idx = sorted(gpu_cells)
    with ThreadPoolExecutor(max_workers=host_threads()) as ex:
        ok = list(ex.map(one, idx))
    return {"sets": len(idx), "points": int(sum(sets[k].shape[0] for k in idx)), "equal": all(ok),
            "mismatched_sets": [k for k, o in zip(idx, ok) if not o][:10],
            "method": "the reference build (oracle/_ref) of every "
                       f"{every}th set, canonical order, against the timed build's cells"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle

    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
        return 0
    sets = workload_sets(args.sets, 0, gen=oracle)
    sample = cpu_sample(sets)
    threads = host_threads()
    times, pts = [], 0
    for step in range(args.warmup + args.steps):
        wall, _, pts = reference_build_sets(sample, threads)
        if step >= args.warmup:
            times.append(wall)
    value = pts * len(times) / sum(times)
    cfg = config(args.sets, sum(a.shape[0] for a in sets))
    desc = (f"every {CPU_EVERY}th set of the workload per step ({len(sample)} sets, {pts} points), "
            f"one set per thread on {threads} host threads (each reference build is single-threaded)")
    cfg["reference_sample"] = desc
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "points/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfg,
            "cpu_baseline": {"value": value, "unit": "points/s", "cores": threads,
                             "kind": "reference", "sample": desc},
            "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---- ours ----------------------------------------------------------------------------


# Measured DRAM traffic of the insertion kernel per point it inserts, from a
# one-kernel ncu capture: dram__bytes_read.sum + dram__bytes_write.sum of the
# fast variant's launch at the finest level of a 256-set case of this workload
# (8.40 GB + 5.77 GB), over the 1,069,032 points that launch inserted.  Traffic
# per inserted point stays the same at full size: every insertion does the same
# kind of work on a tet table much larger than L2.
INSERT_DRAM_BYTES_PER_POINT = 13249.0
# Algorithmic bytes of the build per point: the coordinates read (24 B) plus the
# finite tets written (6.75 per point x 16 B).
BUILD_BYTES_PER_POINT = 24.0 + 6.75 * 16.0


def plain_leg(torch, d3, x, offs, stream, out, sets_idx):
    """The plain one-set-per-call path over the sets `sets_idx` (device-resident
    slices of the batch input).  Returns per-set (points, ms)."""
    handle = stream.cuda_stream
    res = []
    with torch.cuda.stream(stream):
        for k in sets_idx[:8]:                         # warm-up calls
            a, b = int(offs[k]), int(offs[k + 1])
            d3.build_device(x[a:b], out=out, stream=handle)
        torch.cuda.synchronize()
        for k in sets_idx:
            a, b = int(offs[k]), int(offs[k + 1])
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            d3.build_device(x[a:b], out=out, stream=handle)
            e1.record(stream)
            e1.synchronize()
            res.append((b - a, e0.elapsed_time(e1)))
    return res


def plain_1e7_leg(torch, d3, dev, stream, run_ref):
    import oracle

    host = d3.gen_uniform(PLAIN_N, PLAIN_SEED)
    x = torch.from_numpy(host).to(dev)
    out = torch.empty((8 * PLAIN_N + 64, 4), dtype=torch.int32, device=dev)
    handle = stream.cuda_stream
    ms = []
    with torch.cuda.stream(stream):
        d3.build_device(x, out=out, stream=handle)
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            cells, _ = d3.build_device(x, out=out, stream=handle)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
    ncells = int(cells.shape[0])
    del x, out, cells
    torch.cuda.empty_cache()
    r = {"points": PLAIN_N, "ms": min(ms), "points_per_s": PLAIN_N / (min(ms) / 1000.0),
         "tets": ncells}
    if run_ref and oracle.ref_available():
        sample = host[:REF_PLAIN_SAMPLE].copy()
        nc = ctypes.c_int64(0)
        t = oracle.ref().ref_build_time(sample.ctypes.data, sample.shape[0], ctypes.byref(nc))
        r["reference_points_per_s_1thread"] = REF_PLAIN_SAMPLE / t
        r["reference_sample"] = (f"first {REF_PLAIN_SAMPLE:.0e} of the same points, one thread "
                                 f"({t:.2f} s; the reference build is single-threaded)")
        r["gpu_over_reference"] = r["points_per_s"] / r["reference_points_per_s_1thread"]
    return r


SERVING_RATES = (25, 50, 100, 150)     # requests/s
SERVING_SECONDS = 4.0
SERVING_POOL = 160


def serving_leg(torch, d3):
    """Poisson request streams through d3.Server, one per rate."""
    import numpy as np

    pool = d3.mixed_workload(SERVING_POOL, lo=100, hi=1_000_000, seed=31, first_seed=7000)
    pinned = []
    for a in pool:
        t = torch.empty(a.shape, dtype=torch.float64).pin_memory()
        t.numpy()[:] = a
        pinned.append(t.numpy())
    sizes = np.array([a.shape[0] for a in pool])
    out = []
    with d3.Server() as srv:
        for t in [srv.submit(pinned[k]) for k in range(8)]:       # warm-up
            srv.wait(t)
        for rate in SERVING_RATES:
            rng = np.random.default_rng(rate)
            n_req = int(rate * SERVING_SECONDS)
            arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
            picks = rng.integers(0, SERVING_POOL, n_req)
            tickets = []
            t0 = time.perf_counter()
            for a, k in zip(arrivals, picks):
                dt = t0 + a - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                tickets.append(srv.submit(pinned[k]))
            res = [srv.wait(t) for t in tickets]
            lat = [1000.0 * (r.t_done - r.t_submit) for r in res]
            span = max(r.t_done for r in res) - min(r.t_submit for r in res)
            pts = int(sizes[picks].sum())
            out.append({"rate_req_per_s": rate, "requests": n_req, "points": pts,
                        "points_per_s": pts / span, "requests_per_s": n_req / span,
                        "latency_ms_p50": pct(lat, 50), "latency_ms_p99": pct(lat, 99),
                        "mean_batch_sets": float(np.mean([r.batch_sets for r in res]))})
        st = srv.stats()
    return {"sweep": out, "slots": st["slots"], "hbm_budget_bytes": st["hbm_budget_bytes"],
            "peak_bytes_in_use": st["peak_bytes_in_use"],
            "workload": f"Poisson arrivals, {SERVING_SECONDS:.0f} s of arrivals per rate; each request "
                        f"one of {SERVING_POOL} pre-generated sets (sizes log-uniform in [100, 1e6], "
                        "uniform / 8-cluster / lattice / quantised sphere), pinned host memory; "
                        "latency = submit to cells on the host"}


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

    t_gen = time.perf_counter()
    sets = rank_sets(args.sets, rank, world, args.scaling)
    t_gen = time.perf_counter() - t_gen
    sizes = np.array([a.shape[0] for a in sets], dtype=np.int64)
    offs = np.zeros(len(sets) + 1, dtype=np.int64)
    offs[1:] = np.cumsum(sizes)
    n = int(offs[-1])
    pinned = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    pin_np = pinned.numpy()
    np.concatenate(sets, out=pin_np)
    x = pinned.to(dev)
    out = torch.empty((8 * n + 64 * len(sets), 4), dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    handle = stream.cuda_stream

    chunk = args.chunk or None          # None: the device default (tuned below)
    tuning = None
    if not args.no_autotune and not args.profile_run:
        # Setup, not timed: time the candidate speed settings on a 1-in-8 sample
        # of the sets and make the fastest this device's default.
        sample = sets[::8]
        soff = np.zeros(len(sample) + 1, dtype=np.int64)
        soff[1:] = np.cumsum([a.shape[0] for a in sample])
        xs = torch.from_numpy(np.concatenate(sample)).to(dev)
        tuning = d3.autotune(xs, soff, stream=handle)
        tuning["sample"] = f"every 8th set ({len(sample)} sets, {int(soff[-1])} points)"
        del xs

    def step(stats=None, timing=False):
        if timing:
            return _timed_batch(d3, x, offs, out, handle, chunk, stats)
        return d3.build_batch_device(x, offs, out=out, stream=handle, chunk=chunk, stats=stats)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()

    # ---- timed region: device-resident inputs ----
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(gpu_id(torch, dev)) if rank == 0 else None
    # One event between consecutive steps: their differences give each step's
    # time, the first and last the timed region's.
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    e0, e1 = evs[0], evs[-1]
    e0.record(stream)
    ncells = 0
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            cells, co, nv = step()
            ncells = int(cells.shape[0])
            evs[k + 1].record(stream)
    torch.cuda.synchronize()
    step_ms = sorted(evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps))
    clk = clocks.stop() if clocks else None
    # After the timed region: the cells of a sample of sets, for the parity check.
    # Every rank checks the sets it built (their parity is combined below).
    par_cells = None
    if not args.no_cpu_baseline and not args.profile_run:
        every = args.parity_every or PARITY_EVERY
        par_cells = {k: cells[int(co[k]):int(co[k + 1])].cpu().numpy() for k in range(0, len(sets), every)}
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1) / args.steps
    value, s_max, _ = job_rate(dist, dev, n, ms / 1000.0)
    tets_rate, _, _ = job_rate(dist, dev, ncells, ms / 1000.0)
    ms_max = s_max * 1000.0

    if args.profile_run:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
                              "config": config(len(sets), n), "cells": ncells, "profile_run": True}))
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    # ---- instrumented (untimed) step: per-kernel times and live counts ----
    stats = {}
    with torch.cuda.stream(stream):
        step(stats=stats, timing=True)
    torch.cuda.synchronize()
    launches_per_step = count_launches(torch, lambda: step())

    # ---- end to end through the host C ABI d3g_build_batch ----
    lib = d3.library()
    opts = d3._Options()
    lib.d3g_options_default(ctypes.byref(opts))
    if args.chunk:
        opts.chunk = int(args.chunk)

    def e2e_call():
        res = d3._BatchResult()
        d3._check(lib.d3g_build_batch(pin_np.ctypes.data, offs.ctypes.data, len(sets),
                                      ctypes.byref(opts), ctypes.byref(res)), "build_batch")
        total = int(res.cell_offsets[len(sets)])
        lib.d3g_batch_result_free(ctypes.byref(res))
        return total

    e2e_value, e2e_cells = None, 0
    if not args.no_e2e:
        e2e_call()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_cells = e2e_call()
        t_e2e = (time.perf_counter() - t0) / args.steps
        e2e_value, _, _ = job_rate(dist, dev, n, t_e2e)

    # ---- the plain one-set-per-call path on a sample of the same sets ----
    plain = None
    if not args.no_plain:
        idx = list(range(0, len(sets), PLAIN_EVERY))
        per = plain_leg(torch, d3, x, offs, stream, out, idx)
        pts = sum(p for p, _ in per)
        tot_ms = sum(m for _, m in per)
        lat = [m for _, m in per]
        plain = {"points_per_s": pts / (tot_ms / 1000.0),
                 "sample": f"every {PLAIN_EVERY}th set ({len(idx)} sets, {pts} points), "
                           "one d3g_build_device call per set, device-resident input",
                 "latency_ms_p50": pct(lat, 50), "latency_ms_p99": pct(lat, 99),
                 "latency_ms_max": max(lat)}
        plain["batched_over_plain"] = (n / (ms / 1000.0)) / plain["points_per_s"]

    line = None
    if rank == 0:
        peaks, peak_kind = measured_peaks()
        hbm = float(peaks.get("hbm_gbs", HBM_FALLBACK_GBS))
        # Dominant insertion kernel and its algorithmic bytes (C, F: conflict-
        # region tets and boundary facets, counted live, split between the
        # asynchronous passes and the rounds in proportion to the points each
        # inserted).  An insertion must read the vertex record (16 B) and the
        # lock or claim word (4 / 8 B) of every region and ring tet and the
        # neighbour record (16 B) of every region tet; the asynchronous pass
        # also writes the new tets (32 B each, one per boundary facet) and the
        # outside tets' back pointers (4 B each).
        kern = {"k_insert_async": stats.get("ms_async", 0.0), "k_cavity": stats.get("ms_cavity", 0.0),
                "k_check": stats.get("ms_check", 0.0), "k_restar": stats.get("ms_restar", 0.0)}
        dom = max(kern, key=kern.get)
        C, F = stats.get("region_tets", 0), stats.get("boundary_facets", 0)
        inserted = max(1, n - len(sets))
        share = min(1.0, stats.get("async_inserted", 0) / inserted)
        if dom == "k_insert_async":
            Ca, Fa = C * share, F * share
            model_bytes = 20 * (Ca + Fa) + 16 * Ca + 36 * Fa
            launches = max(1, stats.get("launches_async", 1))
            units = stats.get("async_inserted", 0)
        else:
            Cr, Fr = C * (1 - share), F * (1 - share)
            model_bytes = {"k_cavity": 24 * (Cr + Fr) + 16 * Cr, "k_check": 8 * (Cr + Fr) + 16 * Fr,
                           "k_restar": 32 * Cr + 32 * Fr + 40 * Fr}[dom]
            launches = max(1, stats.get("launches_cavity", 1))
            units = inserted - stats.get("async_inserted", 0)
        sec_per_launch = kern[dom] / launches / 1000.0 if kern[dom] else 0.0
        # The survey's algorithmic bytes: 132 B per point the kernel inserts.
        alg_bytes = BUILD_BYTES_PER_POINT * units / launches
        achieved = alg_bytes / sec_per_launch / 1e9 if sec_per_launch else 0.0
        model_achieved = (model_bytes / launches) / sec_per_launch / 1e9 if sec_per_launch else 0.0
        traffic = INSERT_DRAM_BYTES_PER_POINT * units / launches if dom == "k_insert_async" else None
        line = {
            "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
            "higher_is_better": True, "scaling": args.scaling if world > 1 else "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": dict(config(len(sets), n), **({"partition": f"{args.sets} sets split among {world} ranks "
                                                                   "by estimated cost n log2 n"}
                                                    if world > 1 and args.scaling == "strong" else {})),
            "tets_per_s": tets_rate,
            "step_ms": {"min": step_ms[0], "median": step_ms[len(step_ms) // 2], "max": step_ms[-1],
                        "note": "this rank's device time of each timed step"},
            "e2e": ({"value": e2e_value, "unit": "points/s", "h2d_bytes_per_step": 24 * n,
                     "d2h_bytes_per_step": 16 * int(e2e_cells) + 16 * len(sets) + 8}
                    if e2e_value else None),
            "plain": plain,
            "latency": {"batched_set_ms_p50": ms, "batched_set_ms_p99": ms,
                        "note": "a batched set completes with its batch; plain = one call per set",
                        "plain_set_ms_p50": plain["latency_ms_p50"] if plain else None,
                        "plain_set_ms_p99": plain["latency_ms_p99"] if plain else None},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                         "traffic": traffic,
                         "bytes_per_launch": alg_bytes, "points_per_launch": units / launches,
                         "ms_per_launch": kern[dom] / launches,
                         "bytes_definition": f"{BUILD_BYTES_PER_POINT:.0f} B per inserted point (24 B of "
                                             "coordinates in, 6.75 finite tets x 16 B out)",
                         "traffic_definition": f"{INSERT_DRAM_BYTES_PER_POINT:.0f} DRAM bytes per inserted "
                                               "point measured by ncu x the points per launch",
                         "builder_model": {"achieved": model_achieved, "frac": model_achieved / hbm,
                                           "bytes_per_launch": model_bytes / launches,
                                           "definition": "20 B per region and ring tet read (vertices "
                                                         "+ lock), 16 B per region tet's neighbours, "
                                                         "36 B per new tet written"}},
            "gpu_launches": (launches_per_step * args.steps) if launches_per_step else None,
            "clocks": clk,
            "build_stats": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in stats.items()},
            "cells": ncells, "generate_s": round(t_gen, 2), "tuning": tuning,
        }
    if dist:
        dist.barrier()
    # Parity on every rank, over its own sets; with several ranks the outcome is
    # combined (every rank takes part in the same reduction) and any mismatch
    # fails the run on every rank.
    parity = None
    if par_cells is not None:
        parity = parity_leg(sets, par_cells, args.parity_every or PARITY_EVERY)
        if dist:
            flags = torch.tensor([0.0 if parity is None else float(not parity["equal"]),
                                  0.0 if parity is None else float(parity["sets"]),
                                  0.0 if parity is None else float(parity["points"])],
                                 dtype=torch.float64, device=dev)
            dist.all_reduce(flags, op=dist.ReduceOp.SUM)
            if parity is not None:
                parity = dict(parity, ranks=world, sets=int(flags[1].item()), points=int(flags[2].item()),
                              equal=flags[0].item() == 0.0,
                              mismatched_sets=parity["mismatched_sets"] if rank == 0 else [])
    if rank == 0 and world == 1:
        if not args.no_plain:
            line["plain_1e7"] = plain_1e7_leg(torch, d3, dev, stream, not args.no_cpu_baseline)
        if not args.no_serving:
            line["serving"] = serving_leg(torch, d3)
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_leg(sets)
    if rank == 0 and parity is not None:
        line["parity"] = parity
    if rank == 0:
        # The figures of the headline metric, last in the line.
        srv = (line.get("serving") or {}).get("sweep") or []
        p1e7 = line.get("plain_1e7") or {}
        line["headline"] = {
            "batched_points_per_s": value,
            "e2e_points_per_s": e2e_value,
            "plain_points_per_s": plain["points_per_s"] if plain else None,
            "batched_over_plain": plain["batched_over_plain"] if plain else None,
            "e2e_over_plain": (e2e_value / plain["points_per_s"]) if plain and e2e_value else None,
            "plain_set_ms_p50": plain["latency_ms_p50"] if plain else None,
            "plain_set_ms_p99": plain["latency_ms_p99"] if plain else None,
            "serving_ms_p50_by_rate": {str(r["rate_req_per_s"]): r["latency_ms_p50"] for r in srv},
            "serving_ms_p99_by_rate": {str(r["rate_req_per_s"]): r["latency_ms_p99"] for r in srv},
            "plain_1e7_over_reference_1thread": p1e7.get("gpu_over_reference"),
            "parity_equal": (line.get("parity") or {}).get("equal"),
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if parity is not None and not parity["equal"]:
        if rank == 0:
            print("bench: the timed build's cells differ from the reference's", file=sys.stderr)
        return 1
    return 0


def _timed_batch(d3, x, offs, out, handle, chunk, stats):
    """One batched build with per-kernel event timing (slower; untimed)."""
    import numpy as np

    lib = d3.library()
    nsets = offs.shape[0] - 1
    co = np.zeros(nsets + 1, dtype=np.int64)
    nv = np.zeros(nsets, dtype=np.int64)
    opts = d3._Options()
    lib.d3g_options_default(ctypes.byref(opts))
    if chunk:
        opts.chunk = int(chunk)
    opts.timing = 1
    st = d3.BuildStats()
    d3._check(lib.d3g_build_batch_device(x.data_ptr(), offs.ctypes.data, nsets, ctypes.byref(opts),
                                         out.data_ptr(), out.shape[0], co.ctypes.data, nv.ctypes.data,
                                         ctypes.c_void_p(handle), ctypes.byref(st)), "build_batch_device")
    stats.update(st.as_dict())


# ---- microbenchmarks: predicates and spatial sort ------------------------------------

PRED_POINTS = 10_000_000
PRED_QUERIES = 100_000_000
PRED_DEGENERATE = 0.10
ORIENT3D_OPS, IN_SPHERE_OPS = 32, 111      # separate FP64 add/sub/mul of each filter


def lattice_sphere_vectors(n2):
    """Every integer vector (x, y, z) with x^2 + y^2 + z^2 = n2."""
    import numpy as np

    import math

    r = math.isqrt(n2)
    x, y = np.meshgrid(np.arange(-r, r + 1), np.arange(-r, r + 1), indexing="ij")
    z2 = n2 - x * x - y * y
    ok = z2 >= 0
    x, y, z2 = x[ok], y[ok], z2[ok]
    z = np.floor(np.sqrt(z2.astype(np.float64))).astype(np.int64)
    z += (z + 1) * (z + 1) <= z2          # exact integer square root
    z -= z * z > z2
    hit = z * z == z2
    x, y, z = x[hit], y[hit], z[hit]
    v = np.concatenate([np.stack([x, y, z], 1), np.stack([x, y, -z], 1)[z > 0]])
    return v


def predicate_inputs(seed=2):
    """Point table: 1e7 uniform in [-1,1]^3 (mt19937 seed 2), then groups of
    points exactly degenerate by construction on a 2^-20 grid: 4 points on a
    common lattice plane (orient3d) and 5 points on a common integer-lattice
    sphere of squared radius 1221025 (= 1105^2, many representations) about a
    grid-aligned centre (in_sphere).  Returns (points, n_uniform, plane_base,
    n_plane_groups, sphere_base, n_sphere_groups)."""
    import numpy as np

    import del3d_b200 as d3

    uni = d3.gen_uniform(PRED_POINTS, seed, -1.0, 1.0)
    rng = np.random.default_rng(seed)
    g4 = PRED_POINTS // 40
    a = rng.integers(-2, 3, (g4, 1))
    b = rng.integers(-2, 3, (g4, 1))
    k = rng.integers(-(1 << 17), 1 << 17, (g4, 1))
    i = rng.integers(-(1 << 17), 1 << 17, (g4, 4))
    j = rng.integers(-(1 << 17), 1 << 17, (g4, 4))
    plane = np.stack([i, j, k - a * i - b * j], axis=2).reshape(-1, 3) * 2.0 ** -20
    vecs = lattice_sphere_vectors(1105 * 1105)
    g5 = PRED_POINTS // 50
    centre = rng.integers(-(1 << 19), 1 << 19, (g5, 1, 3))
    pick = np.stack([rng.choice(len(vecs), 5, replace=False) for _ in range(64)])
    sphere = (centre + vecs[pick[rng.integers(0, 64, g5)]]).reshape(-1, 3) * 2.0 ** -20
    pts = np.ascontiguousarray(np.concatenate([uni, plane, sphere]))
    return pts, PRED_POINTS, PRED_POINTS, g4, PRED_POINTS + 4 * g4, g5


def predicate_queries(torch, dev, k, n_uniform, base, groups, n_q, seed):
    """n_q index tuples of arity k on the device: 90% uniform random points,
    10% one degenerate group each (rotated so the degenerate point order varies)."""
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    idx = torch.randint(0, n_uniform, (n_q, k), device=dev, dtype=torch.int32, generator=g)
    n_deg = int(n_q * PRED_DEGENERATE)
    rows = torch.randint(0, n_q, (n_deg,), device=dev, generator=g)
    grp = torch.randint(0, groups, (n_deg, 1), device=dev, generator=g)
    rot = torch.randint(0, k, (n_deg, 1), device=dev, generator=g)
    col = (torch.arange(k, device=dev).view(1, k) + rot) % k
    idx[rows] = (base + grp * k + col).to(torch.int32)
    return idx.contiguous()


def run_predicates(args):
    import numpy as np
    import torch

    import del3d_b200 as d3

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    addmul, fma = d3.fp64_throughput(1 << 17, stream.cuda_stream)
    pts_h, n_uni, pbase, g4, sbase, g5 = predicate_inputs()
    pts = torch.from_numpy(pts_h).to(dev)
    lib = d3.library()
    res = {}
    parity_ok = True
    nq = args.queries or PRED_QUERIES
    for kind, name, k, base, groups, ops in ((d3.ORIENT3D, "orient3d", 4, pbase, g4, ORIENT3D_OPS),
                                             (d3.IN_SPHERE, "in_sphere", 5, sbase, g5, IN_SPHERE_OPS)):
        idx = predicate_queries(torch, dev, k, n_uni, base, groups, nq, 7 + k)
        out = torch.empty(nq, dtype=torch.int8, device=dev)
        st = d3._PredStats()

        def call():
            d3._check(lib.d3g_predicates_device(pts.data_ptr(), pts.shape[0], idx.data_ptr(), nq,
                                                kind, out.data_ptr(), ctypes.c_void_p(stream.cuda_stream),
                                                ctypes.byref(st)), name)

        for _ in range(args.warmup):
            call()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            call()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        qps = nq / (ms / 1000.0)
        signs = torch.bincount((out.to(torch.int16) + 1).cpu(), minlength=3).tolist()
        res[name] = {"queries": nq, "ms": ms, "queries_per_s": qps,
                     "exact_fraction": st.n_exact / nq,
                     "fp64_ops_per_query": ops, "fp64_ops_per_s": qps * ops,
                     "fp64_frac_of_measured_addmul_peak": qps * ops / addmul,
                     "signs_neg_zero_pos": signs}
        if not args.no_cpu_baseline:
            # Sign parity, after the timed calls: a strided sample of the timed
            # stream, plus one query on every degenerate group, against the
            # reference's predicate and the reference's integer oracle.
            sample_idx = idx[::PRED_SAMPLE_STRIDE].cpu().numpy()
            sample_got = out[::PRED_SAMPLE_STRIDE].cpu().numpy()
            grp = np.arange(groups, dtype=np.int64)
            rot = grp % k
            gidx = (base + grp[:, None] * k + (np.arange(k)[None, :] + rot[:, None]) % k).astype(np.int32)
            gidx_d = torch.from_numpy(gidx).to(dev)
            gout = torch.empty(groups, dtype=torch.int8, device=dev)
            d3._check(lib.d3g_predicates_device(pts.data_ptr(), pts.shape[0], gidx_d.data_ptr(), groups, kind,
                                                gout.data_ptr(), ctypes.c_void_p(stream.cuda_stream),
                                                ctypes.byref(st)), name)
            torch.cuda.synchronize()
            res[name]["parity"] = predicate_parity(pts_h, name, [(sample_idx, sample_got),
                                                                  (gidx, gout.cpu().numpy())])
            res[name]["parity"]["sample"] = (f"every {PRED_SAMPLE_STRIDE}th query of the timed stream "
                                             f"({sample_idx.shape[0]}) plus one query per degenerate group "
                                             f"({groups}, point order rotated)")
            parity_ok = parity_ok and res[name]["parity"]["equal"]
        del idx, out
    line = {"metric": "predicate queries/s (filter + exact stage + perturbation)",
            "value": 2 * nq / sum(r["ms"] / 1000.0 for r in res.values()),
            "unit": "queries/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"1e8 orient3d + 1e8 in_sphere over a table of 1e7 points uniform in "
                                   f"[-1,1]^3 plus exactly degenerate groups on a 2^-20 grid "
                                   f"({PRED_DEGENERATE:.0%} of queries): lattice planes (orient3d), "
                                   f"integer-lattice spheres (in_sphere)",
                       "l2": "index arrays 1.6-2 GB per kind (larger than L2)"},
            "fp64_peak": {"addmul_ops_per_s": addmul, "dfma_per_s": fma,
                          "note": "measured here by d3g_microbench_fp64"},
            "predicates": res}
    if not args.no_cpu_baseline:
        line["parity"] = parity_ok
    print(json.dumps(line))
    return 0 if parity_ok else 1


PRED_SAMPLE_STRIDE = 100


def predicate_parity(pts, name, batches):
    """Signs the GPU gave (`batches`: (index tuples, signs) pairs) against the
    reference's predicate (oracle/_ref) and its integer oracle tests/exact.h,
    evaluated on host threads.  None when the reference is absent."""
    import numpy as np

    import oracle

    if not oracle.ref_available():
        return {"equal": True, "checked": 0, "note": "reference not built: not checked"}
    kind = "in_sphere" if name == "in_sphere" else "orient3d"
    idx = np.concatenate([b[0] for b in batches])
    got = np.concatenate([b[1] for b in batches])
    pieces = np.array_split(np.arange(idx.shape[0]), host_threads() * 4)

    def one(fn, part):
        return fn(kind, pts, idx[part])

    with ThreadPoolExecutor(max_workers=host_threads()) as ex:
        ref = np.concatenate(list(ex.map(lambda pt: one(oracle.ref_predicate, pt), pieces)))
        exact = np.concatenate(list(ex.map(lambda pt: one(oracle.exact_predicate, pt), pieces)))
    return {"equal": bool(np.array_equal(got, ref) and np.array_equal(got, exact)), "checked": int(idx.shape[0]),
            "differ_from_reference": int(np.count_nonzero(got != ref)),
            "differ_from_exact": int(np.count_nonzero(got != exact)),
            "zero_signs": int(np.count_nonzero(got == 0))}


def run_plain(args):
    """One plain single-set build of --n points of --dist per step (mt19937 seed 6)."""
    import torch

    import del3d_b200 as d3

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    x = torch.from_numpy(d3.gen_set(args.dist, args.n, PLAIN_SEED)).to(dev)
    n = x.shape[0]
    out = torch.empty((8 * n + 64, 4), dtype=torch.int32, device=dev)
    stats = {}
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            d3.build_device(x, out=out, stream=stream.cuda_stream, timing=args.timing,
                            schedule=args.schedule)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            cells, _ = d3.build_device(x, out=out, stream=stream.cuda_stream, timing=args.timing,
                                       stats=stats, schedule=args.schedule)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    print(json.dumps({"metric": "plain single-set build points/s", "value": n / (ms / 1000.0),
                      "unit": "points/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": ms, "timing": bool(args.timing), "cells": int(cells.shape[0]),
                      "config": {"workload": f"{n} points, {args.dist} (seed {PLAIN_SEED})",
                                 "schedule": "rounds" if args.schedule == 1 else "asynchronous"},
                      "build_stats": {k: (round(v, 3) if isinstance(v, float) else v)
                                      for k, v in stats.items()}}))
    return 0


# The plain single-set configurations: (name, distribution, points, seed).
C3_CONFIGS = (("uniform_1e6", "uniform", 1_000_000, 4),
              ("lattice_100^3", "lattice", 1_000_000, 0),
              ("sphere_1e6_q1024_dedup", "sphere", 1_000_000, 5),
              ("uniform_1e7", "uniform", 10_000_000, 6))


def run_c3(args):
    """The four plain single-set configurations: each built on the GPU through
    d3g_build_device (device-resident input, CUDA events, --warmup untimed then
    --steps timed builds), then its cells compared with the reference's build of
    the same points (oracle/_ref, canonical order).  The reference builds run on
    host threads while the GPU works; each is single-threaded, and its time is
    reported beside the GPU's.  Exits 1 if any set of cells differs."""
    import numpy as np
    import torch

    import del3d_b200 as d3
    import oracle

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    inputs = [(name, d3.gen_set(dist, n, seed)) for name, dist, n, seed in C3_CONFIGS]
    check = oracle.ref_available() and not args.no_cpu_baseline

    def ref_one(pts):
        t0 = time.perf_counter()
        r = oracle.ref_build(pts)
        t = time.perf_counter() - t0
        return oracle.canonical_cells(r["cells"]), int(r["n_vertices"]), t

    pool = ThreadPoolExecutor(max_workers=len(inputs)) if check else None
    futures = [pool.submit(ref_one, pts) for _, pts in inputs] if check else None
    rows, all_equal = [], True
    for k, (name, pts) in enumerate(inputs):
        x = torch.from_numpy(pts).to(dev)
        n = x.shape[0]
        out = torch.empty((8 * n + 64, 4), dtype=torch.int32, device=dev)
        ms = []
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                d3.build_device(x, out=out, stream=stream.cuda_stream)
            torch.cuda.synchronize()
            for _ in range(args.steps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                cells, nv = d3.build_device(x, out=out, stream=stream.cuda_stream)
                e1.record(stream)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
        got = cells.cpu().numpy()
        row = {"config": name, "points": int(n), "ms_median": statistics.median(ms), "ms_min": min(ms),
               "points_per_s": n / (statistics.median(ms) / 1000.0), "tets": int(got.shape[0]),
               "n_vertices": int(nv)}
        if check:
            want, ref_nv, t_ref = futures[k].result()
            equal = bool(got.shape == want.shape and np.array_equal(got, want) and ref_nv == nv)
            all_equal = all_equal and equal
            row.update({"reference_tets": int(want.shape[0]), "parity": equal,
                        "reference_s_1thread": t_ref, "gpu_over_reference": t_ref / (row["ms_median"] / 1000.0)})
        rows.append(row)
        del x, out, cells
        torch.cuda.empty_cache()
    if pool:
        pool.shutdown()
    line = {"metric": "plain single-set build points/s at bit-exact tet sets", "unit": "points/s",
            "value": rows[-1]["points_per_s"], "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "plain single-set builds: 1e6 uniform [0,1)^3 (seed 4), the 100^3 integer "
                                   "lattice, 1e6 unit-sphere samples quantised to 2^-10 with duplicates removed "
                                   "(seed 5), 1e7 uniform (seed 6); value = the 1e7 build",
                       "reference": "oracle/_ref (the reference compiled from source), one thread per build, "
                                    "the four running concurrently on host threads while the GPU builds"},
            "builds": rows, "parity": (all_equal if check else None)}
    print(json.dumps(line))
    return 0 if all_equal else 1


SORT_N = 10_000_000


def run_sort(args):
    import torch

    import del3d_b200 as d3
    import oracle

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    host = d3.gen_uniform(SORT_N, 3)
    x = torch.from_numpy(host).to(dev)
    order = torch.empty(SORT_N, dtype=torch.int32, device=dev)
    lib = d3.library()

    def call():
        d3._check(lib.d3g_spatial_sort_device(x.data_ptr(), SORT_N, order.data_ptr(),
                                              ctypes.c_void_p(stream.cuda_stream)), "spatial_sort")

    for _ in range(args.warmup):
        call()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        call()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    peaks, peak_kind = measured_peaks()
    hbm = float(peaks.get("hbm_gbs", HBM_FALLBACK_GBS))
    gbs = 28.0 * SORT_N / (ms / 1000.0) / 1e9
    line = {"metric": "spatial sort points/s (bit-exact reference order)", "value": SORT_N / (ms / 1000.0),
            "unit": "points/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "1e7 points uniform in [0,1)^3 (mt19937 seed 3)"},
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                         "peak_kind": peak_kind, "bytes_per_point": 28}}
    if oracle.ref_available() and not args.no_cpu_baseline:
        import numpy as np

        o = np.zeros(SORT_N, dtype=np.int32)
        t0 = time.perf_counter()
        oracle.ref().ref_spatial_sort(host.ctypes.data, SORT_N, o.ctypes.data)
        t = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": SORT_N / t, "unit": "points/s", "cores": 1, "kind": "reference",
                                "sample": f"the whole 1e7 points, one thread ({t:.2f} s)"}
        line["order_equals_reference"] = bool(np.array_equal(o, order.cpu().numpy()))
    print(json.dumps(line))
    return 0


READER_EVERY = 16


def _write_reader_files(root, sets):
    """Set k goes to a file in format k % 4: text, binary PLY, OBJ, OFF."""
    import numpy as np

    paths = []
    for k, pts in enumerate(sets):
        fmt = k % 4
        if fmt == 0:
            p = os.path.join(root, f"s{k}.xyz")
            np.savetxt(p, pts, fmt="%.17g")
        elif fmt == 1:
            p = os.path.join(root, f"s{k}.ply")
            hdr = (f"ply\nformat binary_little_endian 1.0\nelement vertex {pts.shape[0]}\n"
                   "property double x\nproperty double y\nproperty double z\nend_header\n").encode()
            with open(p, "wb") as fh:
                fh.write(hdr + np.ascontiguousarray(pts, dtype="<f8").tobytes())
        elif fmt == 2:
            p = os.path.join(root, f"s{k}.obj")
            np.savetxt(p, pts, fmt="v %.17g %.17g %.17g")
        else:
            p = os.path.join(root, f"s{k}.off")
            np.savetxt(p, pts, fmt="%.17g", header=f"OFF\n{pts.shape[0]} 0 0", comments="")
        paths.append(p)
    return paths


def run_readers(args):
    import shutil
    import tempfile

    import numpy as np

    import del3d_b200 as d3

    threads = os.cpu_count() or 1
    sets = workload_sets(args.sets, 0)[::READER_EVERY]
    root = tempfile.mkdtemp(prefix="d3g_readers_")
    try:
        paths = _write_reader_files(root, sets)
        n_points = sum(int(a.shape[0]) for a in sets)
        mb = sum(os.path.getsize(p) for p in paths) / 1e6
        for _ in range(args.warmup):
            d3.load_point_sets(paths, threads=threads)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            xyz, offs, dropped = d3.load_point_sets(paths, threads=threads)
        dt = (time.perf_counter() - t0) / args.steps
        line = {"metric": "input reader points/s (files to back-to-back host points)",
                "value": n_points / dt, "unit": "points/s", "n_gpus": 0, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": f"every {READER_EVERY}th set of the batched workload ({len(sets)} sets, "
                                       f"{n_points} points, {mb:.0f} MB) as files, formats in turn: x y z "
                                       "text, binary little-endian PLY, OBJ, OFF", "threads": threads},
                "sets_equal_input": bool(all(np.array_equal(xyz[offs[k]:offs[k + 1]], a)
                                             for k, a in enumerate(sets)))}
        try:
            import oracle

            ref_ok = oracle.ref_meshio_available()
        except ImportError:
            ref_ok = False
        if ref_ok and not args.no_cpu_baseline:
            with ThreadPoolExecutor(threads) as ex:
                t0 = time.perf_counter()
                ref = list(ex.map(oracle.ref_mesh_load, paths))
                t = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": n_points / t, "unit": "points/s", "cores": threads,
                                    "kind": "reference",
                                    "sample": f"the same {len(paths)} files, one reader call per file on "
                                              f"{threads} host threads ({t:.2f} s)"}
            line["equals_reference"] = bool(all(
                np.array_equal(xyz[offs[k]:offs[k + 1]].view(np.uint64), r[0].view(np.uint64)) and not r[2]
                for k, r in enumerate(ref)))
        print(json.dumps(line))
    finally:
        shutil.rmtree(root, ignore_errors=True)
    return 0


def main():
    args = parse_args()
    if args.workload == "readers":
        return run_readers(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "predicates":
        return run_predicates(args)
    if args.workload == "sort":
        return run_sort(args)
    if args.workload == "plain":
        return run_plain(args)
    if args.workload == "c3":
        return run_c3(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
