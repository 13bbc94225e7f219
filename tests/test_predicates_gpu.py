"""Device predicates vs the oracle, the reference and tests/exact.h: bit-exact signs."""
import numpy as np
import pytest

import del3d_b200 as d3
import oracle

pytestmark = pytest.mark.gpu

CASES = {
    "cylinder": lambda: oracle.ps_cylinder(400, 8),
    "sphere": lambda: oracle.ps_sphere(400, 8),
    "torus": lambda: oracle.ps_torus(400, 8),
    "box": lambda: oracle.ps_box_shell(6),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_quantised_5tuples(cuda, name):
    # The reference's own stage-2 stream (tests/test_predicates.cpp:107-129).
    pts = CASES[name]()
    idx = oracle.ps_rng_below(12345, len(pts), 5 * 20000).reshape(-1, 5).astype(np.int32)
    o4 = d3.orient3d(pts, idx[:, :4])
    assert (o4 == oracle.ref_predicate("orient3d", pts, idx[:, :4])).all()
    assert (o4 == oracle.exact_predicate("orient3d", pts, idx[:, :4])).all()
    for kind, fn in (("in_sphere", d3.in_sphere), ("in_sphere_unperturbed", d3.in_sphere_unperturbed)):
        got = fn(pts, idx)
        assert (got == oracle.ref_predicate(kind, pts, idx)).all(), kind
        assert (got == oracle.orc_predicate(kind, pts, idx)).all(), kind


def test_hand_known_signs(cuda):
    # tests/test_predicates.cpp:58-76: unit corner tetrahedron.
    pts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.25, 0.25, 0.25], [5, 5, 5]], float)
    assert d3.orient3d(pts, [[0, 1, 2, 3]])[0] == 1
    assert d3.orient3d(pts, [[0, 2, 1, 3]])[0] == -1
    assert d3.in_sphere(pts, [[0, 1, 2, 3, 4]])[0] == 1
    assert d3.in_sphere(pts, [[0, 1, 2, 3, 5]])[0] == -1


def test_lattice_degeneracies(cuda):
    # tests/test_predicates.cpp:79-104: constructed ties on a 5^3 lattice.
    base = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [0, 0, 1], [-1, 0, 0], [0, -1, 0]]
    lat = [[i, j, k] for i in range(-2, 3) for j in range(-2, 3) for k in range(-2, 3)]
    rot = [[j, k, i] for i, j, k in lat]
    pts = np.array(base + lat + rot, float)
    nb, nl = len(base), len(lat)
    o_idx = np.array([[0, 1, 2, nb + t] for t in range(nl)], np.int32)
    s_idx = np.array([[1, 2, 4, nb + t, nb + nl + t] for t in range(nl)], np.int32)
    assert (d3.orient3d(pts, o_idx) == oracle.exact_predicate("orient3d", pts, o_idx)).all()
    ok = oracle.ref_predicate("orient3d", pts, s_idx[:, :4]) > 0
    got = d3.in_sphere(pts, s_idx)
    assert (got == oracle.ref_predicate("in_sphere", pts, s_idx)).all()
    assert (got[ok] == oracle.exact_predicate("in_sphere", pts, s_idx)[ok]).all()


def test_random_and_wide_exponents(cuda):
    rng = np.random.default_rng(5)
    pts = np.concatenate([rng.uniform(-1, 1, (2000, 3)),
                          rng.uniform(-1, 1, (500, 3)) * 2.0 ** rng.integers(-60, 60, (500, 1)),
                          np.round(rng.uniform(-1, 1, (500, 3)) * 2 ** 20) / 2 ** 20])
    idx = rng.integers(0, len(pts), (50000, 5)).astype(np.int32)
    for kind, fn in (("orient3d", d3.orient3d), ("in_sphere", d3.in_sphere),
                     ("in_sphere_unperturbed", d3.in_sphere_unperturbed)):
        ii = idx[:, :4] if kind == "orient3d" else idx
        assert (fn(pts, ii) == oracle.ref_predicate(kind, pts, ii)).all(), kind


def test_coplanar_family(cuda):
    # tests/test_predicates2.cpp: z=0 grid, tilted grid z=x+y, cocircular ring.
    rng = np.random.default_rng(11)
    g = np.array([[i, j, 0.0] for i in range(-3, 4) for j in range(-3, 4)] +
                 [[i, j, float(i + j)] for i in range(-3, 4) for j in range(-3, 4)] +
                 [[5, 0, 0], [4, 3, 0], [3, 4, 0], [0, 5, 0], [-3, 4, 0], [-4, 3, 0], [-5, 0, 0],
                  [-4, -3, 0], [-3, -4, 0], [0, -5, 0], [3, -4, 0], [4, -3, 0], [9, 9, 0]], float)
    planes = [np.arange(0, 49), np.arange(49, 98), np.concatenate([np.arange(98, 111), [24]])]
    idx = np.concatenate([p[rng.integers(0, len(p), (20000, 4))] for p in planes]).astype(np.int32)
    col = d3.collinear(g, idx[:, :3])
    assert (col == oracle.ref_predicate("collinear", g, idx[:, :3])).all()
    ok = col == 0
    assert (d3.coplanar_orientation(g, idx[ok, :3]) ==
            oracle.ref_predicate("coplanar_orientation3", g, idx[ok, :3])).all()
    assert (d3.coplanar_orientation(g, idx[ok]) ==
            oracle.ref_predicate("coplanar_orientation4", g, idx[ok])).all()
    for kind, fn in (("coplanar_in_circle", d3.coplanar_in_circle),
                     ("coplanar_in_circle_unperturbed", d3.coplanar_in_circle_unperturbed)):
        assert (fn(g, idx[ok]) == oracle.ref_predicate(kind, g, idx[ok])).all(), kind


def test_orient2d(cuda):
    rng = np.random.default_rng(2)
    six = np.round(rng.uniform(-4, 4, (20000, 6)) * 4) / 4
    six[::3, 4:] = six[::3, :2] + 2 * (six[::3, 2:4] - six[::3, :2])   # collinear third point
    assert (d3.orient2d(six) == np.array(
        [np.sign(np.round((q[2] - q[0]) * (q[5] - q[1]) - (q[3] - q[1]) * (q[4] - q[0]), 12)) for q in six],
        np.int8)).all()


def test_empty_and_invalid(cuda):
    pts = np.zeros((4, 3))
    assert d3.orient3d(pts, np.zeros((0, 4), np.int32)).shape == (0,)
    with pytest.raises(d3.Del3dError):
        d3.orient3d(pts, np.array([[0, 1, 2, 7]], np.int32))   # index out of range


def test_lattice_sphere_groups_2m20(cuda):
    """The predicate microbenchmark's degenerate groups: 5 points on a common
    integer-lattice sphere of squared radius 1105^2 about a grid-aligned centre,
    scaled by 2^-20 (exactly cospherical: the in_sphere tie-break decides), and
    4 points on a common lattice plane (orient3d exactly zero), every rotation
    of the point order."""
    from bench import lattice_sphere_vectors

    rng = np.random.default_rng(21)
    vecs = lattice_sphere_vectors(1105 * 1105)
    assert len(vecs) > 100 and (np.sum(vecs.astype(np.int64) ** 2, axis=1) == 1105 * 1105).all()
    g5 = 400
    centre = rng.integers(-(1 << 19), 1 << 19, (g5, 1, 3))
    pick = np.stack([rng.choice(len(vecs), 5, replace=False) for _ in range(g5)])
    sphere = ((centre + vecs[pick]).reshape(-1, 3) * 2.0 ** -20)
    g4 = 400
    a, b = rng.integers(-2, 3, (g4, 1)), rng.integers(-2, 3, (g4, 1))
    k = rng.integers(-(1 << 17), 1 << 17, (g4, 1))
    i, j = rng.integers(-(1 << 17), 1 << 17, (g4, 4)), rng.integers(-(1 << 17), 1 << 17, (g4, 4))
    plane = np.stack([i, j, k - a * i - b * j], axis=2).reshape(-1, 3) * 2.0 ** -20
    pts = np.concatenate([sphere, plane])
    s_idx = np.concatenate([(np.arange(g5)[:, None] * 5 + (np.arange(5)[None, :] + r) % 5)
                            for r in range(5)]).astype(np.int32)
    o_idx = np.concatenate([(5 * g5 + np.arange(g4)[:, None] * 4 + (np.arange(4)[None, :] + r) % 4)
                            for r in range(4)]).astype(np.int32)
    got = d3.in_sphere(pts, s_idx)
    assert (got != 0).all()
    assert (got == oracle.ref_predicate("in_sphere", pts, s_idx)).all()
    assert (got == oracle.exact_predicate("in_sphere", pts, s_idx)).all()
    assert (d3.in_sphere_unperturbed(pts, s_idx) == 0).all()
    o = d3.orient3d(pts, o_idx)
    assert (o == 0).all() and (o == oracle.ref_predicate("orient3d", pts, o_idx)).all()
