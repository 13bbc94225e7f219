"""Failure paths of the build, forced from the host by lowering a limit
(d3g_options): each must end the call with its status - never a hang, a trap
or corrupt cells - and the next build on the same device must still equal the
reference.  Every limit here is a bounded loop or a capacity check on the
device that records a status word the host reads; nothing faults the GPU.
The reference has no error channel (it grows without bound and aborts only
under DEL3D_VALIDATE, src/triangulation.cpp:110-118); its walk budget is
src/triangulation.cpp:368-369."""
import numpy as np
import pytest

import del3d_b200 as d3
import oracle

pytestmark = pytest.mark.gpu


def _expect(status, pts, **limits):
    import torch

    x = torch.from_numpy(pts).to("cuda")
    with pytest.raises(d3.Del3dError) as e:
        d3.build_device(x, **limits)
    assert e.value.status == status, (e.value, limits)


def _still_correct():
    """A normal build right after the failure equals the reference."""
    pts = d3.gen_lattice(20 ** 3)
    d = d3.Delaunay()
    d.build(pts)
    want = oracle.canonical_cells(oracle.ref_build(pts)["cells"])
    assert np.array_equal(d.finite_cells(), want)


@pytest.mark.parametrize("schedule", [0, 1])
def test_round_limit(cuda, schedule):
    # Lockstep rounds go out 16 to a batch: a limit of 1 is hit by the first batch
    # (schedule 1), or by the first batch the asynchronous pass's leftovers need.
    pts = d3.gen_lattice(20_000)
    if schedule == 0:
        _expect(d3.ERR_ROUND_LIMIT, pts, schedule=0, max_rounds=1, walk_limit=1)
    else:
        _expect(d3.ERR_ROUND_LIMIT, pts, schedule=1, max_rounds=1)
    _still_correct()


@pytest.mark.parametrize("schedule", [0, 1])
def test_tet_capacity(cuda, schedule):
    # One tet slot per vertex where uniform input needs about 6.75: the table
    # fills and the build reports it instead of writing past it.
    _expect(d3.ERR_OOM, d3.gen_uniform(20_000, 3), schedule=schedule, tet_capacity=1)
    _still_correct()


@pytest.mark.parametrize("schedule", [0, 1])
def test_walk_limit(cuda, schedule):
    # One step per walk: the asynchronous attempts give up and leave their points
    # to the rounds, whose walks then stop at the limit with a status.
    _expect(d3.ERR_WALK_LIMIT, d3.gen_uniform(20_000, 3), schedule=schedule, walk_limit=1)
    _still_correct()


@pytest.mark.parametrize("schedule", [0, 1])
def test_cavity_capacity(cuda, schedule):
    # Two region tets per worker, in the normal and the big-round scratch alike:
    # a region that outgrows the big-round scratch reports its status.
    _expect(d3.ERR_CAVITY_CAPACITY, d3.gen_uniform(20_000, 3), schedule=schedule, cavity_capacity=2)
    _still_correct()


def _wide_octahedron(k):
    """The unit octahedron's vertices with one moved off the sphere by 2^-k in
    x: in_sphere calls on it are uncertain for the filter, and their exact
    values span about k binades."""
    pts = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [-1, 0, 0], [0, 0, -1], [0, -1, 0]], dtype=np.float64)
    pts[4, 0] = 2.0 ** -k
    return pts


def test_wide_exact_tier_predicates(cuda):
    """Calls whose exact value needs more than the exact stage's 16 limbs (in_sphere
    over more than about 200 binades, orient3d over more than about 330) go to the
    wide tier and get the exact sign: the octahedron moved off its sphere by 2^-k
    up to k = 1074, nearly cospherical groups spanning 310 binades, and random
    points with exponents in [-200, 200], against the reference's integer oracle
    tests/exact.h, and against the reference's own predicates wherever its
    floating-point expansions cannot underflow or overflow.  (Where they do -
    products of coordinates below 2^-1074, e.g. the octahedron moved by 2^-548 or
    less - the reference's sign is not the exact one; this library's is.  Where
    the filters' own arithmetic overflows or underflows, a filter decision can
    be wrong, the reference's and this library's alike, since the filters are
    the same.)"""
    idx = np.array([[0, 1, 2, 3, 4]], np.int32)
    for k in list(range(200, 1071, 29)) + [1074]:
        pts = _wide_octahedron(k)
        for kind, fn in (("in_sphere", d3.in_sphere), ("in_sphere_unperturbed", d3.in_sphere_unperturbed)):
            got = fn(pts, idx)
            assert (got == oracle.exact_predicate(kind, pts, idx)).all(), (kind, k)
            if 2 * k <= 1074:
                assert (got == oracle.ref_predicate(kind, pts, idx)).all(), (kind, k)
    rng = np.random.default_rng(31)
    # Exponents in [-200, 200]: spans of up to 400 binades, no under/overflow in
    # the reference's degree-5 expansions.
    pts = rng.uniform(-1, 1, (3000, 3)) * 2.0 ** rng.integers(-200, 200, (3000, 1))
    pts[::7, 1] = 0.0
    q = rng.integers(0, len(pts), (20000, 5)).astype(np.int32)
    for kind, fn, ii in (("orient3d", d3.orient3d, q[:, :4]), ("in_sphere", d3.in_sphere, q),
                         ("in_sphere_unperturbed", d3.in_sphere_unperturbed, q)):
        got = fn(pts, ii)
        assert (got == oracle.ref_predicate(kind, pts, ii)).all(), kind
        assert (got[:2000] == oracle.exact_predicate(kind, pts, ii[:2000])).all(), kind
    # Nearly cospherical calls that need the wide tier: five points of an integer
    # lattice sphere (squared radius 1105^2) scaled by 2^s, the fifth moved by
    # 2^(s-300) - every call uncertain for the filter, spanning about 310 binades.
    from bench import lattice_sphere_vectors

    vecs = lattice_sphere_vectors(1105 * 1105).astype(np.float64)
    with_zero = vecs[(vecs == 0).any(axis=1)]
    groups = []
    for g in range(200):
        sc = float(rng.integers(100, 190))
        p5 = vecs[rng.choice(len(vecs), 5, replace=False)] * 2.0 ** sc
        p5[4] = with_zero[rng.integers(0, len(with_zero))] * 2.0 ** sc
        z = int(np.flatnonzero(p5[4] == 0)[0])
        p5[4, z] = (1.0 if g % 2 else -1.0) * 2.0 ** (sc - 300)   # off the sphere by 2^(2s-600)
        groups.append(p5)
    near = np.concatenate(groups)
    qn = (np.arange(200)[:, None] * 5 + np.arange(5)[None, :]).astype(np.int32)
    for kind, fn in (("in_sphere", d3.in_sphere), ("in_sphere_unperturbed", d3.in_sphere_unperturbed)):
        got = fn(near, qn)
        assert (got != 0).all()
        assert (got == oracle.exact_predicate(kind, near, qn)).all(), kind
        assert (got == oracle.ref_predicate(kind, near, qn)).all(), kind
    # Points on a plane through the origin tilted by 2^-800: orient3d exactly
    # resolvable only with about 2400 bits.
    plane = np.array([[1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0], [2.0 ** -800, 0.5, 0.5]])
    o = np.array([[0, 1, 2, 3], [1, 0, 2, 3]], np.int32)
    assert (d3.orient3d(plane, o) == oracle.exact_predicate("orient3d", plane, o)).all()


def test_exact_capacity_build(cuda):
    _expect(d3.ERR_EXACT_CAPACITY, _wide_octahedron(250))
    _still_correct()
    ok = _wide_octahedron(200)
    d = d3.Delaunay()
    d.build(ok)
    assert np.array_equal(d.finite_cells(), oracle.canonical_cells(oracle.ref_build(ok)["cells"]))


@pytest.mark.parametrize("dist", ["uniform", "clusters", "lattice", "sphere"])
@pytest.mark.parametrize("schedule", [0, 1])
def test_validate_after_every_level(cuda, dist, schedule):
    """The device port of the reference's Tds::validate() (src/tds.h:483-530),
    run after every BRIO level, finds nothing wrong, and the cells are the same
    as without it."""
    import torch

    pts = d3.gen_set(dist, 30_000, 41)
    x = torch.from_numpy(pts).to(cuda)
    stats = {}
    a, nv = d3.build_device(x, schedule=schedule, validate=True, stats=stats)
    a = a.clone()
    b, nv2 = d3.build_device(x, schedule=schedule)
    assert nv == nv2 and torch.equal(a, b)
    # The per-build counters: every insertion made conflict tests; lattices need
    # tie-breaks, uniform points none.
    assert stats["conflict_tests"] > 10 * len(pts)
    assert stats["max_region_tets"] >= 1
    if dist == "lattice":
        assert stats["tie_breaks"] > 0 and stats["uncertain_tests"] >= stats["tie_breaks"]
    if dist == "uniform":
        assert stats["tie_breaks"] == 0


def test_validate_batched(cuda):
    import torch

    sets = d3.mixed_workload(64, 32, 8000, seed=5, first_seed=900)
    offs = np.zeros(len(sets) + 1, dtype=np.int64)
    offs[1:] = np.cumsum([len(a) for a in sets])
    x = torch.from_numpy(np.concatenate(sets)).to(cuda)
    a, co, nv = d3.build_batch_device(x, offs, validate=True)
    a = a.clone()
    b, co2, nv2 = d3.build_batch_device(x, offs)
    assert (co == co2).all() and (nv == nv2).all() and torch.equal(a, b)
