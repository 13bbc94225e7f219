"""Batched builds: every set of a mixed batch equals its single-set build and the
reference's canonical tet set."""
import numpy as np
import pytest

import del3d_b200 as d3
import oracle

pytestmark = pytest.mark.gpu


def mixed_sets():
    rng = np.random.default_rng(17)
    sets = [
        d3.gen_uniform(3000, 1),
        oracle.ps_lattice(7, 7, 7),
        d3.gen_clusters(2500, 3),
        d3.gen_sphere(4000, 5, q=64, dedupe=False),             # duplicates
        np.array([[i, j, 0.0] for i in range(6) for j in range(6)]),   # coplanar: no cells
        np.zeros((0, 3)),                                       # empty
        np.array([[i, 2.0 * i, 3.0 * i] for i in range(9)]),    # collinear
        np.tile([1.0, 2.0, 3.0], (5, 1)),                       # one distinct point
        rng.integers(0, 5, (400, 3)).astype(np.float64),        # duplicate grid
        np.array([[i, j, 0.0] for i in range(6) for j in range(6)] + [[2.0, 2.0, 3.0]]),
        oracle.ps_box_shell(5),
        d3.gen_uniform(17, 4),
        d3.gen_uniform(70000, 9),                               # several BRIO levels
    ]
    return sets


def test_mixed_batch_matches_single_and_reference(cuda):
    sets = mixed_sets()
    cells, nv = d3.build_batch(sets)
    assert len(cells) == len(sets)
    for k, pts in enumerate(sets):
        r = oracle.ref_build(pts) if len(pts) else {"cells": np.zeros((0, 4), np.int32), "n_vertices": 0}
        want = oracle.canonical_cells(r["cells"])
        assert nv[k] == r["n_vertices"], k
        assert cells[k].shape == want.shape and (cells[k] == want).all(), k


def test_batch_equals_repeated_plain(cuda):
    sets = d3.mixed_workload(40, lo=32, hi=5000, seed=5)
    cells, nv = d3.build_batch(sets)
    for k, pts in enumerate(sets):
        d = d3.Delaunay()
        d.build(pts)
        assert (cells[k] == d.finite_cells()).all() and nv[k] == d.number_of_vertices(), k


def test_batch_device_entry(cuda):
    import torch

    sets = d3.mixed_workload(12, lo=32, hi=3000, seed=7)
    offs = np.zeros(len(sets) + 1, dtype=np.int64)
    offs[1:] = np.cumsum([len(a) for a in sets])
    x = torch.from_numpy(np.concatenate(sets)).cuda()
    cells, co, nv = d3.build_batch_device(x, offs)
    host, hnv = d3.build_batch(sets)
    allc = cells.cpu().numpy()
    for k in range(len(sets)):
        assert (allc[co[k]:co[k + 1]] == host[k]).all() and nv[k] == hnv[k]
