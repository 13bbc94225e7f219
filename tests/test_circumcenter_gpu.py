"""Device circumcentres against the reference's del3d::circumcenter and
del3d::circumcenter_lazy (src/triangulation.cpp:805-930), compiled from its own
sources.

Tolerance (stated in include/del3d_b200.h): per coordinate,
|ours - reference| <= 4 ulp(|reference - p0|) + 1 ulp(|reference|); the two
are bit-identical whenever the reference's expansion sum rounds to the nearest
double, so the tests also require (almost) every coordinate to be identical.
"""
import numpy as np
import pytest

import del3d_b200 as d3
import oracle

pytestmark = pytest.mark.gpu

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


def _within_bound(ours, ref, p0):
    q = np.abs(ref - p0)
    tol = 4 * np.spacing(q) + np.spacing(np.abs(ref))
    return np.abs(ours - ref) <= tol


def _compare(pts, tets, lazy, min_identical=0.999):
    ours = d3.circumcenters(pts, tets, lazy=lazy)
    ref = oracle.ref_circumcenters(pts, tets, lazy=lazy)
    p0 = pts[tets[:, 0]]
    same = (ours == ref) | (np.isnan(ours) & np.isnan(ref))
    ok = same | _within_bound(ours, ref, p0)
    assert ok.all(), (f"{(~ok).sum()} coordinates outside the bound, e.g. tet "
                      f"{np.argwhere(~ok)[0][0]}: ours {ours[~ok][:3]} ref {ref[~ok][:3]}")
    assert same.mean() >= min_identical, f"only {same.mean():.6f} bit-identical"
    return same.mean()


def _sliver_tets(rng, n):
    """Four points within 1e-9 of a common plane: the denominator cancels."""
    base = rng.uniform(0, 1, (n, 3, 3))
    w = rng.uniform(0, 1, (n, 3))
    w /= w.sum(axis=1, keepdims=True)
    p3 = np.einsum("nk,nkd->nd", w, base) + rng.normal(0, 1e-9, (n, 3))
    pts = np.concatenate([base, p3[:, None, :]], axis=1).reshape(-1, 3)
    return pts, np.arange(4 * n, dtype=np.int32).reshape(n, 4)


@needs_ref
@pytest.mark.parametrize("lazy", [False, True])
def test_delaunay_cells_uniform(cuda, lazy):
    pts = d3.gen_uniform(20000, 11)
    d = d3.Delaunay()
    d.build(pts, all_cells=False, incident=False)
    _compare(pts, d.finite_cells(), lazy)


@needs_ref
@pytest.mark.parametrize("lazy", [False, True])
def test_random_tets_full_mantissas(cuda, lazy):
    rng = np.random.default_rng(5)
    pts = np.concatenate([d3.gen_clusters(3000, 3), rng.normal(0, 1, (3000, 3))])
    tets = rng.integers(0, len(pts), (50000, 4)).astype(np.int32)
    _compare(pts, tets, lazy)


@needs_ref
@pytest.mark.parametrize("lazy", [False, True])
def test_slivers(cuda, lazy):
    pts, tets = _sliver_tets(np.random.default_rng(7), 20000)
    _compare(pts, tets, lazy)
    if lazy:
        d3.circumcenters(pts, tets, lazy=True)
        n, n_exact = d3.predicate_stats()
        assert n == tets.shape[0] and n_exact > 0      # slivers reach the exact fallback


@needs_ref
@pytest.mark.parametrize("lazy", [False, True])
def test_lattice_and_coplanar(cuda, lazy):
    pts = d3.gen_lattice(1000).astype(np.float64)
    rng = np.random.default_rng(9)
    tets = rng.integers(0, len(pts), (30000, 4)).astype(np.int32)
    ours = d3.circumcenters(pts, tets, lazy=lazy)
    ref = oracle.ref_circumcenters(pts, tets, lazy=lazy)
    assert (ours == ref).all()
    # coplanar tets (one lattice plane) give their first vertex
    flat = np.flatnonzero(pts[:, 2] == 3.0)
    ct = rng.choice(flat, (100, 4)).astype(np.int32)
    got = d3.circumcenters(pts, ct, lazy=lazy)
    assert (got == pts[ct[:, 0]]).all()


@needs_ref
@pytest.mark.parametrize("lazy", [False, True])
def test_wide_exponent_span(cuda, lazy):
    rng = np.random.default_rng(13)
    scale = 10.0 ** rng.integers(-20, 20, (4000, 1))
    pts = rng.uniform(-1, 1, (4000, 3)) * scale
    tets = rng.integers(0, len(pts), (20000, 4)).astype(np.int32)
    _compare(pts, tets, lazy)


@needs_ref
def test_single_tet_api(cuda):
    a, b, c, d = (0.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0)
    p = d3.circumcenter(a, b, c, d)
    assert (p.x, p.y, p.z) == (0.5, 0.5, 0.5)
    q = d3.circumcenter_lazy(a, b, c, d)
    assert (q.x, q.y, q.z) == (0.5, 0.5, 0.5)


def test_index_out_of_range(cuda):
    pts = np.zeros((4, 3))
    with pytest.raises(d3.Del3dError):
        d3.circumcenters(pts, [[0, 1, 2, 4]])
