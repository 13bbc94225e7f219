"""The device block cache under the library's buffers: blocks of 1 MiB and
more that a call frees serve later calls on any stream (after an event that
marks the end of their last use), so a repeated build draws nothing new from
the stream-ordered pool.  Cells must not depend on which block a buffer got
(tolerance: none - tet sets are integers)."""
import numpy as np
import pytest

import del3d_b200 as d3

pytestmark = pytest.mark.gpu


def _cells(pts):
    d = d3.Delaunay()
    d.build(pts, all_cells=False, incident=False)
    return d.finite_cells()


def test_repeated_build_reuses_cached_blocks(cuda):
    pts = d3.gen_uniform(400_000, 21)
    first = _cells(pts)
    _cells(pts)
    used0, _ = d3.pool_usage(reset_high=True)
    again = _cells(pts)
    used1, high = d3.pool_usage()
    assert np.array_equal(again, first)
    # Only blocks under 1 MiB come from the pool; 1600 B/point would be 640 MB.
    assert high - used0 <= 64 << 20, (used0, high)
    assert abs(used1 - used0) <= 64 << 20, (used0, used1)


def test_blocks_move_between_streams(cuda):
    import torch

    sets = [d3.gen_uniform(200_000, 31), d3.gen_clusters(150_000, 32), d3.gen_lattice(120_000)]
    want = [_cells(p) for p in sets]
    streams = [torch.cuda.Stream() for _ in range(3)]
    for rep in range(2):
        for k, p in enumerate(sets):
            s = streams[(k + rep) % 3]
            x = torch.from_numpy(p.astype(np.float64)).cuda()
            torch.cuda.synchronize()
            cells, nv = d3.build_device(x, stream=s.cuda_stream)
            assert np.array_equal(cells.cpu().numpy(), want[k]), (rep, k)


def test_release_returns_cached_blocks(cuda):
    d3.release_cached_memory()
    base, _ = d3.pool_usage()
    _cells(d3.gen_uniform(300_000, 41))
    cached, _ = d3.pool_usage()
    assert cached - base >= 100 << 20, (base, cached)      # the build's blocks wait in the cache
    d3.release_cached_memory()
    after, _ = d3.pool_usage()
    assert after <= base, (base, cached, after)
    assert np.array_equal(_cells(d3.gen_uniform(5000, 3)), _cells(d3.gen_uniform(5000, 3)))
