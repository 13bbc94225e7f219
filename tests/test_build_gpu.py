"""The device build vs the reference compiled from source and the oracle:
canonical tet sets bit-exact, vertex counts, all_cells, incident_cells."""
import numpy as np
import pytest

import del3d_b200 as d3
import oracle

pytestmark = pytest.mark.gpu

CASES = {
    "random5": lambda: oracle.ps_random_cube(5, 4),
    "random8": lambda: oracle.ps_random_cube(8, 4),
    "random20": lambda: oracle.ps_random_cube(20, 4),
    "random100": lambda: oracle.ps_random_cube(100, 4),
    "random500": lambda: oracle.ps_random_cube(500, 4),
    "lattice5": lambda: oracle.ps_lattice(5, 5, 5),
    "plane_apex": lambda: np.array([[i, j, 0.0] for i in range(6) for j in range(6)] + [[2.0, 2.0, 3.0]]),
    "box5": lambda: oracle.ps_box_shell(5),
    "cylinder": lambda: oracle.ps_cylinder(300),
    "sphere": lambda: oracle.ps_sphere(300),
    "torus": lambda: oracle.ps_torus(300),
    "lattice12": lambda: oracle.ps_lattice(12, 12, 12),
    "uniform20k": lambda: d3.gen_uniform(20000, 1),
    "sphere_q1024": lambda: d3.gen_sphere(20000, 5),
    "clusters": lambda: d3.gen_clusters(20000, 7),
    # Duplicates: a repeated point keeps the index of its copy that comes last in
    # the reference's spatial order (src/triangulation.cpp:77-81).
    "dup_grid": lambda: np.random.default_rng(3).integers(0, 6, (3000, 3)).astype(np.float64),
    "dup_copies": lambda: np.concatenate([d3.gen_uniform(5000, 2), d3.gen_uniform(5000, 2)[::3],
                                          -np.zeros((7, 3)), np.zeros((5, 3))]),
    "sphere_q_dups": lambda: d3.gen_sphere(30000, 5, q=64, dedupe=False),
    # The centre of a sphere, first: every cell holds it, so its canonical bucket
    # holds all cells (sorted by one block at 300 points, by the radix sort of
    # every cell beyond 2048 cells).
    "sphere_centre300": lambda: np.concatenate([np.zeros((1, 3)), oracle.ps_sphere(300)]),
    "sphere_centre3000": lambda: np.concatenate([np.zeros((1, 3)), oracle.ps_sphere(3000)]),
}


def reference(pts):
    r = oracle.ref_build(pts)
    return r, oracle.canonical_cells(r["cells"]), oracle.canonical_cells(r["all"])


@pytest.mark.parametrize("case", sorted(CASES))
def test_cells_match_reference(cuda, case):
    pts = CASES[case]()
    r, cells, allc = reference(pts)
    d = d3.Delaunay()
    d.build(pts)
    assert d.number_of_vertices() == r["n_vertices"]
    got = d.finite_cells()
    assert got.shape == cells.shape and (got == cells).all()
    assert d.all_cells().shape == allc.shape and (d.all_cells() == allc).all()
    # incident_cells agrees with finite_cells (tests/test_delaunay.cpp:141-159).
    inc = d.incident_cells()
    want = [[] for _ in range(len(pts))]
    for ci, t in enumerate(got.tolist()):
        for v in t:
            want[v].append(ci)
    assert all(list(a) == b for a, b in zip(inc, want))


def test_deterministic(cuda):
    pts = d3.gen_uniform(50000, 9)
    a, b = d3.Delaunay(), d3.Delaunay()
    a.build(pts)
    b.build(pts)
    assert (a.finite_cells() == b.finite_cells()).all()


@pytest.mark.parametrize("pts", [np.zeros((0, 3)), np.zeros((1, 3)), np.array([[0, 0, 0], [1, 0, 0.0]]),
                                 np.tile([1.0, 2.0, 3.0], (20, 1)),
                                 np.array([[i, 2.0 * i, 3.0 * i] for i in range(10)]),
                                 np.array([[i, j, 0.0] for i in range(5) for j in range(5)])])
def test_degenerate_inputs_have_no_cells(cuda, pts):
    d = d3.Delaunay()
    d.build(pts)
    assert d.finite_cells().shape[0] == 0
    assert d.number_of_vertices() == len({tuple(p) for p in pts.tolist()})


def test_non_finite_rejected(cuda):
    pts = d3.gen_uniform(100, 1)
    pts[17, 1] = np.nan
    with pytest.raises(d3.Del3dError):
        d3.Delaunay().build(pts)


@pytest.mark.parametrize("dist", ["uniform", "clusters", "lattice", "sphere"])
def test_schedules_and_lane_counts_agree(cuda, dist):
    """The tet set does not depend on the insertion order, so the asynchronous
    lock-based schedule, the lockstep rounds and every lane count must give the
    same canonical cells, bit for bit, on every seed."""
    import torch

    for seed in range(3):
        pts = d3.gen_set(dist, 40000 + 7919 * seed, 100 + seed)
        x = torch.from_numpy(pts).to(cuda)
        base, nv = d3.build_device(x, schedule=0)
        base = base.clone()
        for kw in ({"schedule": 1}, {"schedule": 1, "lanes": 8}, {"schedule": 1, "lanes": 4},
                   {"schedule": 0, "chunk": -12, "alpha_small": 12}):
            other, nv2 = d3.build_device(x, **kw)
            assert nv2 == nv and torch.equal(other, base), (dist, seed, kw)


@pytest.mark.parametrize("case", ["lattice12", "sphere_q1024", "dup_grid", "uniform20k", "box5", "random500"])
def test_level_growth_same_cells(cuda, case):
    """The BRIO level growth of the build's insertion order (the reference's 8,
    or 2-7 for more and shorter levels) changes the order only: the canonical
    cells and the vertex count equal the reference's for every growth."""
    import torch

    pts = CASES[case]()
    r, want, _ = reference(pts)
    x = torch.from_numpy(np.ascontiguousarray(pts)).to(cuda)
    for g in (2, 3, 4, 8):
        cells, nv = d3.build_device(x, level_growth=g)
        got = oracle.canonical_cells(cells.cpu().numpy())
        assert nv == r["n_vertices"] and np.array_equal(got, want), (case, g)


def test_level_growth_out_of_range(cuda):
    import torch

    x = torch.from_numpy(d3.gen_uniform(1000, 3)).to(cuda)
    for g in (1, 9, -2):
        with pytest.raises(d3.Del3dError):
            d3.build_device(x, level_growth=g)
    cells, _ = d3.build_device(x)
    assert cells.shape[0] > 0
