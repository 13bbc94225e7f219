"""The multi-GPU rank logic of bench.py on the CPU: two gloo ranks (world size
2, 127.0.0.1).  With N GPUs every rank builds its own sets - no data-path
collective, sets are independent - and the whole-job rate is the points all
ranks processed over the slowest rank's time.  No GPU is needed."""
import json
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sets = bench.rank_sets(64, rank, world, "weak")
        again = bench.workload_sets(64, rank)
        n = sum(int(a.shape[0]) for a in sets)
        seconds = 1.0 + rank                       # rank 1 is the slow one
        rate, t_max, total = bench.job_rate(dist, torch.device("cpu"), n, seconds)
        # strong scaling: this rank's share of the one shared workload
        full = bench.workload_sets(64, 0)
        mine = bench.rank_sets(64, rank, world, "strong")
        idx = [next(k for k, f in enumerate(full) if f.shape == a.shape and (f == a).all()) for a in mine]
        n_strong = sum(int(a.shape[0]) for a in mine)
        s_rate, s_max, s_total = bench.job_rate(dist, torch.device("cpu"), n_strong, 2.0 - rank)
        # the same collective order on every rank, as in the bench's timed region
        dist.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as fh:
            json.dump({"n": n, "sizes": [int(a.shape[0]) for a in sets], "rate": rate, "t_max": t_max,
                       "total": total, "deterministic": all((a == b).all() for a, b in zip(sets, again)),
                       "strong_idx": idx, "strong_total": s_total, "strong_rate": s_rate,
                       "full_points": sum(int(a.shape[0]) for a in full)}, fh)
    finally:
        dist.destroy_process_group()


def test_two_ranks_build_their_own_sets_and_sum_points(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    r = [json.load(open(tmp_path / f"rank{k}.json")) for k in range(world)]
    assert all(x["deterministic"] for x in r)
    assert r[0]["sizes"] != r[1]["sizes"]                 # each rank its own sets
    total = r[0]["n"] + r[1]["n"]
    assert r[0]["n"] != r[1]["n"]                         # so the job total is a sum, not world * n
    for x in r:
        assert x["t_max"] == 2.0 and x["total"] == total
        assert x["rate"] == pytest.approx(total / 2.0)
    # strong scaling: the two shares are disjoint and together the whole workload
    a, b = set(r[0]["strong_idx"]), set(r[1]["strong_idx"])
    assert not (a & b) and a | b == set(range(64))
    for x in r:
        assert x["strong_total"] == x["full_points"]
        assert x["strong_rate"] == pytest.approx(x["full_points"] / 2.0)


def test_single_rank_rate_needs_no_process_group():
    import torch

    sys.path.insert(0, ROOT)
    import bench

    rate, t_max, total = bench.job_rate(None, torch.device("cpu"), 1000, 0.5)
    assert (rate, t_max, total) == (2000.0, 0.5, 1000.0)


def test_partition_balances_and_covers():
    sys.path.insert(0, ROOT)
    import numpy as np

    import del3d_b200 as d3

    rng = np.random.default_rng(3)
    sizes = np.floor(np.exp(rng.uniform(np.log(32), np.log(65536), 1000))).astype(int)
    for parts_n in (1, 2, 3, 8):
        parts = d3.partition_sets(sizes, parts_n)
        assert sorted(sum(parts, [])) == list(range(1000))
        cost = sizes * np.log2(np.maximum(sizes, 2))
        loads = np.array([cost[p].sum() for p in parts])
        # longest-first greedy: no part exceeds the mean by more than the largest set
        assert loads.max() <= loads.mean() + cost.max()
    assert d3.partition_sets(sizes, 4) == d3.partition_sets(list(sizes), 4)        # deterministic
    w = np.where(np.arange(1000) % 4 == 2, 5.0, 1.0)                              # lattice-like sets cost more
    assert sorted(sum(d3.partition_sets(sizes, 3, w), [])) == list(range(1000))
    with pytest.raises(ValueError):
        d3.partition_sets(sizes, 0)
