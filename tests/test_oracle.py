"""The oracle (our CPU restatement) pinned against the reference: the golden
hashes the reference's own tests hold, and the reference compiled from source."""
import numpy as np
import pytest

import oracle

# tests/test_spatial_sort.cpp:115-147 of the reference: FNV-1a of the order.
SORT_GOLDEN = [(0, 0x14650fb0739d0383), (1, 0x315446a086a23133), (2, 0x29034675a49f07c2),
               (5, 0x744ddb73fb935d27), (8, 0x7ec129e73709cb53), (9, 0x580cd772e82efaab),
               (63, 0x18cf12b455d4e1ac), (64, 0x4fde96ee0b2e8be3), (65, 0xafa28526c6130f43),
               (200, 0x23d15ee1f09fef23), (1000, 0x8b7191bde7a7449b)]

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference not built")


@needs_ref
@pytest.mark.parametrize("n,h", SORT_GOLDEN)
def test_spatial_sort_pinned_random(n, h):
    pts = oracle.ps_random_cube(n, 7)
    assert oracle.fnv1a_order(oracle.orc_spatial_sort(pts)) == h


@needs_ref
@pytest.mark.parametrize("case,h", [
    ("lattice", 0xdb779fbe6eb82833), ("box", 0x1667fe1e40586b6a), ("same", 0xc9325f52533ad94f),
    ("cylinder", 0x0b3b773499c64173), ("sphere", 0x93fb3414e085d46b), ("torus", 0x0e117e42cb5f457f)])
def test_spatial_sort_pinned_degenerate(case, h):
    pts = {"lattice": lambda: oracle.ps_lattice(12, 12, 6), "box": lambda: oracle.ps_box_shell(8),
           "same": lambda: np.tile([1.0, 2.0, 3.0], (300, 1)),
           "cylinder": lambda: oracle.ps_cylinder(2000), "sphere": lambda: oracle.ps_sphere(2000),
           "torus": lambda: oracle.ps_torus(2000)}[case]()
    assert oracle.fnv1a_order(oracle.orc_spatial_sort(pts)) == h


@needs_ref
def test_reference_pinned_cell_hashes():
    # tests/test_delaunay.cpp:208-243 pin the reference's own cell sequence: this
    # checks that oracle/_ref is the real reference.
    for n, h in [(5, 0x5a7aed0478362803), (8, 0x0b63a88c5b428feb), (20, 0xdc8940eebc8963d7),
                 (100, 0x92dcfb61db16f9c3), (500, 0xab8f0ef0a819629a)]:
        assert oracle.fnv1a_cells(oracle.ref_build(oracle.ps_random_cube(n, 4))["cells"]) == h
    assert oracle.fnv1a_cells(oracle.ref_build(oracle.ps_lattice(5, 5, 5))["cells"]) == 0xf0f09ebcc3974328


@needs_ref
@pytest.mark.parametrize("name", ["cylinder", "sphere", "torus", "box"])
def test_predicates_match_reference_and_exact(name):
    pts = {"cylinder": lambda: oracle.ps_cylinder(400, 8), "sphere": lambda: oracle.ps_sphere(400, 8),
           "torus": lambda: oracle.ps_torus(400, 8), "box": lambda: oracle.ps_box_shell(6)}[name]()
    idx = oracle.ps_rng_below(12345, len(pts), 5 * 20000).reshape(-1, 5).astype(np.int32)
    o4 = oracle.orc_predicate("orient3d", pts, idx[:, :4])
    assert (o4 == oracle.ref_predicate("orient3d", pts, idx[:, :4])).all()
    assert (o4 == oracle.exact_predicate("orient3d", pts, idx[:, :4])).all()
    assert (o4 == 0).sum() > 0          # exact ties really were exercised
    for kind in ("in_sphere", "in_sphere_unperturbed"):
        a = oracle.orc_predicate(kind, pts, idx)
        assert (a == oracle.ref_predicate(kind, pts, idx)).all()
        pos = o4 > 0   # exact.h states in_sphere under its precondition only
        assert (a[pos] == oracle.exact_predicate(kind, pts, idx)[pos]).all()


@needs_ref
def test_coplanar_predicates_match_reference():
    rng = np.random.default_rng(11)
    g = np.array([[i, j, 0.0] for i in range(-3, 4) for j in range(-3, 4)] +
                 [[i, j, float(i + j)] for i in range(-3, 4) for j in range(-3, 4)])
    idx = rng.integers(0, 49, size=(20000, 4)).astype(np.int32) + (rng.integers(0, 2, size=(20000, 1)) * 49).astype(np.int32)
    col = oracle.orc_predicate("collinear", g, idx[:, :3])
    assert (col == oracle.ref_predicate("collinear", g, idx[:, :3])).all()
    ok = col == 0
    for kind in ("coplanar_orientation3",):
        assert (oracle.orc_predicate(kind, g, idx[ok, :3]) == oracle.ref_predicate(kind, g, idx[ok, :3])).all()
    for kind in ("coplanar_orientation4", "coplanar_in_circle", "coplanar_in_circle_unperturbed"):
        assert (oracle.orc_predicate(kind, g, idx[ok]) == oracle.ref_predicate(kind, g, idx[ok])).all()


def canon_ref(pts):
    r = oracle.ref_build(pts)
    return oracle.canonical_cells(r["cells"]), oracle.canonical_cells(r["all"]), r["n_vertices"]


CASES = {
    "random500": lambda: oracle.ps_random_cube(500, 4),
    "lattice5": lambda: oracle.ps_lattice(5, 5, 5),
    "plane_apex": lambda: np.array([[i, j, 0.0] for i in range(6) for j in range(6)] + [[2.0, 2.0, 3.0]]),
    "box5": lambda: oracle.ps_box_shell(5),
    "cylinder": lambda: oracle.ps_cylinder(300),
    "sphere": lambda: oracle.ps_sphere(300),
    "torus": lambda: oracle.ps_torus(300),
    "lattice10": lambda: oracle.ps_lattice(10, 10, 10),
    "dup_grid": lambda: np.random.default_rng(3).integers(0, 4, (300, 3)).astype(np.float64),
}


@needs_ref
@pytest.mark.parametrize("case", sorted(CASES))
def test_build_matches_reference(case):
    pts = CASES[case]()
    cells, allc, nv = canon_ref(pts)
    o = oracle.orc_build(pts)
    assert o["n_vertices"] == nv
    assert o["cells"].shape == cells.shape and (o["cells"] == cells).all()
    assert o["all"].shape == allc.shape and (o["all"] == allc).all()


def test_build_degenerate_no_cells():
    for pts in (np.zeros((0, 3)), np.zeros((1, 3)), np.tile([1.0, 2.0, 3.0], (20, 1)),
                np.array([[i, 2.0 * i, 3.0 * i] for i in range(10)], dtype=float),
                np.array([[i, j, 0.0] for i in range(5) for j in range(5)], dtype=float)):
        o = oracle.orc_build(pts)
        assert o["cells"].shape[0] == 0
    assert oracle.orc_build(np.tile([1.0, 2.0, 3.0], (20, 1)))["n_vertices"] == 1


def test_oracle_workload_generators_match_the_library():
    """The reference arm of bench.py draws its inputs from the oracle's copy of
    the point generators (so it never loads libdel3d_b200.so); they must be the
    product library's, bit for bit."""
    import del3d_b200 as d3

    ours = d3.mixed_workload(24, 32, 4096, seed=7, first_seed=300)
    orc = oracle.mixed_workload(24, 32, 4096, seed=7, first_seed=300)
    assert len(ours) == len(orc)
    for a, b in zip(ours, orc):
        assert a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))
    assert np.array_equal(d3.gen_uniform(1000, 6).view(np.uint64), oracle.gen_uniform(1000, 6).view(np.uint64))
