"""The request server (d3g_server_*): continuous batching with admission by a
device-memory budget.

The property that matters: a request's cells are the same whether it is built
alone or mixed with others in a batch, arriving while other batches run
(tolerance: none - tet sets and their canonical order are integers).
"""
import threading
import time

import numpy as np
import pytest

import del3d_b200 as d3
import oracle


def test_server_without_device_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(d3.Del3dError):
        d3.Server()


def _alone(pts):
    d = d3.Delaunay()
    d.build(pts, all_cells=False, incident=False)
    return d.finite_cells(), d.number_of_vertices()


@pytest.mark.gpu
def test_results_equal_alone_and_in_mix(cuda):
    sets = d3.mixed_workload(48, lo=100, hi=200_000, seed=77, first_seed=500)
    results = {}
    with d3.Server(slots=3) as srv:
        # A first wave submitted at once (queued requests are batched), then
        # submitters that keep adding requests while batches are on the GPU.
        tickets = {srv.submit(sets[i]): i for i in range(16)}
        lock = threading.Lock()

        def feeder(idx):
            rng = np.random.default_rng(idx[0])
            for i in idx:
                time.sleep(float(rng.uniform(0, 0.02)))
                t = srv.submit(sets[i])
                with lock:
                    tickets[t] = i

        threads = [threading.Thread(target=feeder, args=(list(range(16 + k, 48, 4)),)) for k in range(4)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        for t, i in list(tickets.items()):
            results[i] = srv.wait(t)
        st = srv.stats()
    assert st["completed"] == 48 and st["queued"] == 0
    assert st["batches"] < 48, st                       # requests shared batches
    assert st["peak_in_flight_requests"] > 1, st
    assert max(r.batch_sets for r in results.values()) > 1
    for i, pts in enumerate(sets):
        cells, nv = _alone(pts)
        r = results[i]
        assert np.array_equal(r.cells, cells), f"request {i} ({pts.shape[0]} points) differs from alone"
        assert r.n_vertices == nv
        assert r.t_submit <= r.t_admit <= r.t_done
    # and alone equals the reference on a few of them
    if oracle.ref_available():
        for i in (0, 5, 11):
            want = oracle.canonical_cells(oracle.ref_build(sets[i])["cells"])
            assert np.array_equal(results[i].cells, want)


@pytest.mark.gpu
def test_admission_respects_budget(cuda):
    sets = [d3.gen_uniform(300_000, 40 + k) for k in range(12)]
    budget = 2 << 30
    with d3.Server(slots=4, hbm_budget_bytes=budget) as srv:
        tickets = [srv.submit(p) for p in sets]
        res = [srv.wait(t) for t in tickets]
        st = srv.stats()
    assert st["peak_bytes_in_use"] <= budget, st
    assert st["batches"] >= 2, st                       # the budget split the work
    for p, r in zip(sets[:3], res[:3]):
        assert np.array_equal(r.cells, _alone(p)[0])


@pytest.mark.gpu
def test_request_larger_than_budget_runs_alone(cuda):
    sets = [d3.gen_uniform(20_000, k) for k in range(6)]
    with d3.Server(slots=3, hbm_budget_bytes=1) as srv:
        res = [srv.wait(t) for t in [srv.submit(p) for p in sets]]
        st = srv.stats()
    assert st["peak_in_flight_requests"] == 1 and st["batches"] == 6, st
    for p, r in zip(sets, res):
        assert np.array_equal(r.cells, _alone(p)[0])


@pytest.mark.gpu
def test_bad_request_fails_alone(cuda):
    good = [d3.gen_uniform(5000, k) for k in range(5)]
    bad = d3.gen_uniform(5000, 99)
    bad[17, 1] = np.nan
    with d3.Server(slots=1) as srv:
        srv_t = [srv.submit(p) for p in good[:2]] + [srv.submit(bad)] + [srv.submit(p) for p in good[2:]]
        out = []
        for t in srv_t:
            try:
                out.append(srv.wait(t))
            except d3.Del3dError as e:
                out.append(e)
    assert isinstance(out[2], d3.Del3dError)
    for p, r in zip(good, out[:2] + out[3:]):
        assert np.array_equal(r.cells, _alone(p)[0])


@pytest.mark.gpu
def test_wait_timeout_and_memory_estimate(cuda):
    # The admission estimate (1600 B/point + 160 MiB per batch) bounds the
    # pool's high-water mark of a build.
    for pts in (d3.gen_uniform(1_000_000, 3), d3.gen_lattice(400_000), d3.gen_clusters(500_000, 2)):
        d3.pool_usage(reset_high=True)
        used0, _ = d3.pool_usage()
        _alone(pts)
        _, high = d3.pool_usage()
        assert high - used0 <= 1600 * pts.shape[0] + (160 << 20), (pts.shape[0], high - used0)
    with d3.Server(slots=1) as srv:
        t = srv.submit(d3.gen_uniform(2_000_000, 5))
        with pytest.raises(TimeoutError):
            srv.wait(t, timeout=0.0)
        assert srv.wait(t).cells.shape[0] > 0
