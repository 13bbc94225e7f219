"""d3g_predicates_noalloc_device: the predicate entry point for callers that
cannot allocate device memory (its scratch is a fixed array of the library).

Its signs must equal those of the allocating entry point d3g_predicates_device
exactly (signs are exact: the tolerance is zero), on two calls in a row - the
second call reuses the array the first one left behind.  Collected last so a
run that stops at the first failure has run everything else already.
"""
import ctypes

import numpy as np
import pytest

import del3d_b200 as d3
import oracle

pytestmark = pytest.mark.gpu

MAX_QUERIES = 1 << 20


def _lib():
    lib = d3.library()
    fn = lib.d3g_predicates_noalloc_device
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return lib


def _run(fn, pts, idx, kind, torch):
    out = torch.zeros(idx.shape[0], dtype=torch.int8, device=pts.device)
    st = fn(pts.data_ptr(), pts.shape[0], idx.data_ptr(), idx.shape[0], kind, out.data_ptr(), None,
            None)
    assert st == 0, d3.library().d3g_last_error().decode()
    return out.cpu().numpy()


def _inputs(torch, dev, seed):
    # Quantised surface samples (many exact ties: the exact-stage queue is used)
    # mixed with generic points.
    rng = np.random.default_rng(seed)
    pts = np.concatenate([oracle.ps_sphere(400, 8, seed), oracle.ps_box_shell(6),
                          rng.uniform(-1, 1, (3000, 3))])
    idx = rng.integers(0, len(pts), (200000, 5)).astype(np.int32)
    return (torch.from_numpy(pts).to(dev), torch.from_numpy(np.ascontiguousarray(idx)).to(dev))


@pytest.mark.parametrize("kind", [d3.ORIENT3D, d3.IN_SPHERE, d3.IN_SPHERE_UNPERTURBED,
                                  d3.COPLANAR_IN_CIRCLE])
def test_noalloc_matches_allocating_entry_point(cuda, kind):
    import torch

    lib = _lib()
    k = lib.d3g_predicate_arity(kind)
    for call, seed in enumerate((1, 2)):          # two calls in a row
        pts, idx5 = _inputs(torch, cuda, seed)
        idx = idx5[:, :k].contiguous()
        got = _run(lib.d3g_predicates_noalloc_device, pts, idx, kind, torch)
        want = _run(lib.d3g_predicates_device, pts, idx, kind, torch)
        assert (got == want).all(), f"call {call}: signs differ from d3g_predicates_device"


def test_noalloc_exact_stage_used_and_counted(cuda):
    import torch

    lib = _lib()
    pts, idx = _inputs(torch, cuda, 3)
    st = (ctypes.c_int64 * 2)()
    out = torch.zeros(idx.shape[0], dtype=torch.int8, device=cuda)
    assert lib.d3g_predicates_noalloc_device(pts.data_ptr(), pts.shape[0], idx.data_ptr(),
                                             idx.shape[0], d3.IN_SPHERE, out.data_ptr(), None,
                                             ctypes.cast(st, ctypes.c_void_p)) == 0
    assert st[0] == idx.shape[0] and st[1] > 0     # some queries reached the exact stage
    ref = oracle.ref_predicate("in_sphere", pts.cpu().numpy(), idx.cpu().numpy())
    assert (out.cpu().numpy() == ref).all()


def test_noalloc_rejects_too_many_queries(cuda):
    import torch

    lib = _lib()
    pts = torch.zeros((8, 3), dtype=torch.float64, device=cuda)
    idx = torch.zeros((4, 5), dtype=torch.int32, device=cuda)
    out = torch.zeros(4, dtype=torch.int8, device=cuda)
    st = lib.d3g_predicates_noalloc_device(pts.data_ptr(), 8, idx.data_ptr(), MAX_QUERIES + 1,
                                           d3.IN_SPHERE, out.data_ptr(), None, None)
    assert st == 1   # D3G_ERR_INVALID_ARGUMENT, before any device work
    assert b"D3G_NOALLOC_MAX_QUERIES" in lib.d3g_last_error()


def test_noalloc_at_the_limit_matches_counts(cuda):
    """Exactly D3G_NOALLOC_MAX_QUERIES in_sphere queries on points of one
    integer-lattice sphere (squared radius 1105^2, scaled by 2^-20): every query
    is exactly cospherical, so every one goes through the exact-stage queue in
    the fixed array, filling it to its last element.  Signs and the exact-stage
    count equal the allocating entry point's."""
    import torch

    from bench import lattice_sphere_vectors

    lib = _lib()
    rng = np.random.default_rng(9)
    pts_h = lattice_sphere_vectors(1105 * 1105).astype(np.float64) * 2.0 ** -20
    idx_h = rng.integers(0, len(pts_h), (MAX_QUERIES, 5)).astype(np.int32)
    pts = torch.from_numpy(pts_h).to(cuda)
    idx = torch.from_numpy(idx_h).to(cuda)
    res = {}
    for name in ("d3g_predicates_noalloc_device", "d3g_predicates_device"):
        st = d3._PredStats()
        out = torch.zeros(MAX_QUERIES, dtype=torch.int8, device=cuda)
        rc = getattr(lib, name)(pts.data_ptr(), pts.shape[0], idx.data_ptr(), MAX_QUERIES, d3.IN_SPHERE,
                                out.data_ptr(), None, ctypes.byref(st))
        assert rc == 0, lib.d3g_last_error().decode()
        res[name] = (out.cpu().numpy(), st.n_queries, st.n_exact)
    got, want = res["d3g_predicates_noalloc_device"], res["d3g_predicates_device"]
    assert got[1] == want[1] == MAX_QUERIES
    assert got[2] == want[2] == MAX_QUERIES, (got[2], want[2])
    assert np.array_equal(got[0], want[0])


def test_noalloc_reports_calls_beyond_the_exact_stage(cuda):
    """The fixed array holds no arena for the wide tier: an in_sphere call whose
    exact value needs more than 16 limbs is reported (D3G_ERR_EXACT_CAPACITY),
    never answered wrongly; the allocating entry point answers it."""
    import torch

    lib = _lib()
    pts_h = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [-1, 0, 0], [2.0 ** -250, 0, -1]], dtype=np.float64)
    pts = torch.from_numpy(pts_h).to(cuda)
    idx = torch.tensor([[0, 1, 2, 3, 4]], dtype=torch.int32, device=cuda)
    out = torch.zeros(1, dtype=torch.int8, device=cuda)
    st = lib.d3g_predicates_noalloc_device(pts.data_ptr(), 5, idx.data_ptr(), 1, d3.IN_SPHERE, out.data_ptr(),
                                           None, None)
    assert st == d3.ERR_EXACT_CAPACITY
    assert _run(lib.d3g_predicates_device, pts, idx, d3.IN_SPHERE, torch)[0] == \
        oracle.ref_predicate("in_sphere", pts_h, np.array([[0, 1, 2, 3, 4]], np.int32))[0]
