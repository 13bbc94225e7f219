"""Parity oracles for the del3d ``Delaunay::build`` path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this
package, and only as the oracle or the timed CPU baseline -- never as part of
the product path (``del3d_b200`` never imports it).

Two libraries are loaded through ctypes:

* ``liboracle.so`` -- our CPU restatement of the reference algorithm
  (``oracle/oracle.cpp``: predicates, rand48 + Hilbert spatial sort, sequential
  Bowyer-Watson build, canonical cell order);
* ``_ref/libdel3d_ref.so`` -- the reference del3d compiled from its own sources
  (``oracle/Makefile``) plus its integer oracle ``tests/exact.h`` and its test
  point-set generators ``tests/pointsets.h``;
* ``_ref/libmeshio_ref.so`` -- the reference viewer's mesh reader
  (``viewer/mesh_io.cpp``) compiled from its source, the oracle of the input
  readers.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORC_PATH = os.path.join(_HERE, "liboracle.so")
_REF_PATH = os.path.join(_HERE, "_ref", "libdel3d_ref.so")

_MESHIO_PATH = os.path.join(_HERE, "_ref", "libmeshio_ref.so")

_orc: Optional[ctypes.CDLL] = None
_ref: Optional[ctypes.CDLL] = None
_meshio: Optional[ctypes.CDLL] = None

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_INT = ctypes.c_int


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def orc() -> ctypes.CDLL:
    global _orc
    if _orc is None:
        lib = ctypes.CDLL(_ORC_PATH)
        for name in ("orc_orient3d", "orc_coplanar_orientation3", "orc_coplanar_orientation4",
                     "orc_collinear"):
            getattr(lib, name).argtypes = [_P, _P, _I64, _P]
        for name in ("orc_in_sphere", "orc_coplanar_in_circle"):
            getattr(lib, name).argtypes = [_P, _P, _I64, _INT, _P]
        lib.orc_orient2d.argtypes = [_P, _I64, _P]
        lib.orc_spatial_sort.argtypes = [_P, _I64, _P]
        lib.orc_shuffle.argtypes = [_I64, _P]
        lib.orc_build.argtypes = [_P, _I64]
        lib.orc_build.restype = _P
        for name in ("orc_build_ncells", "orc_build_nall", "orc_build_nvertices"):
            getattr(lib, name).argtypes = [_P]
            getattr(lib, name).restype = _I64
        lib.orc_build_cells.argtypes = [_P, _P]
        lib.orc_build_all.argtypes = [_P, _P]
        lib.orc_build_free.argtypes = [_P]
        lib.orc_canonical_rotate.argtypes = [_P, _I64]
        lib.d3g_gen_uniform.argtypes = [_I64, ctypes.c_uint32, ctypes.c_double, ctypes.c_double, _P]
        lib.d3g_gen_sphere.argtypes = [_I64, ctypes.c_uint32, ctypes.c_double, ctypes.c_int32, _P]
        lib.d3g_gen_clusters.argtypes = [_I64, ctypes.c_uint32, ctypes.c_int32, ctypes.c_double, _P]
        lib.d3g_gen_lattice.argtypes = [_I64, _P]
        for name in ("d3g_gen_uniform", "d3g_gen_sphere", "d3g_gen_clusters", "d3g_gen_lattice"):
            getattr(lib, name).restype = None
        _orc = lib
    return _orc


def ref_available() -> bool:
    return os.path.exists(_REF_PATH)


def ref() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(_REF_PATH)
        for name in ("ref_orient3d", "ref_coplanar_orientation3", "ref_coplanar_orientation4",
                     "ref_collinear", "exact_orient3d", "exact_coplanar_orientation3",
                     "exact_coplanar_orientation4", "exact_collinear"):
            getattr(lib, name).argtypes = [_P, _P, _I64, _P]
        for name in ("ref_in_sphere", "ref_coplanar_in_circle", "exact_in_sphere",
                     "exact_coplanar_in_circle"):
            getattr(lib, name).argtypes = [_P, _P, _I64, _INT, _P]
        lib.ref_orient2d.argtypes = [_P, _I64, _P]
        lib.ref_spatial_sort.argtypes = [_P, _I64, _P]
        lib.ref_build.argtypes = [_P, _I64]
        lib.ref_build.restype = _P
        for name in ("ref_build_ncells", "ref_build_nall", "ref_build_nvertices"):
            getattr(lib, name).argtypes = [_P]
            getattr(lib, name).restype = _I64
        lib.ref_build_cells.argtypes = [_P, _P]
        lib.ref_build_all.argtypes = [_P, _P]
        lib.ref_build_incident.argtypes = [_P, _P, _P]
        lib.ref_build_incident.restype = _I64
        lib.ref_build_free.argtypes = [_P]
        lib.ref_build_time.argtypes = [_P, _I64, _P]
        lib.ref_build_time.restype = ctypes.c_double
        lib.ref_circumcenter.argtypes = [_P, _P, _I64, _INT, _P]
        for name, args in (("ps_cylinder", [_I64, _INT, ctypes.c_uint, _P]),
                           ("ps_sphere", [_I64, _INT, ctypes.c_uint, _P]),
                           ("ps_torus", [_I64, _INT, ctypes.c_uint, _P]),
                           ("ps_box_shell", [_INT, _P]),
                           ("ps_lattice", [_INT, _INT, _INT, _P]),
                           ("ps_random_cube", [_I64, ctypes.c_uint, _P])):
            getattr(lib, name).argtypes = args
            getattr(lib, name).restype = _I64
        lib.ps_rng_below.argtypes = [ctypes.c_uint, _I64, _I64, _P]
        _ref = lib
    return _ref


# ---- helpers -------------------------------------------------------------------

_ARITY = {"orient3d": 4, "in_sphere": 5, "in_sphere_unperturbed": 5, "coplanar_orientation3": 3,
          "coplanar_orientation4": 4, "coplanar_in_circle": 4,
          "coplanar_in_circle_unperturbed": 4, "collinear": 3}


def _pred(lib: ctypes.CDLL, prefix: str, kind: str, pts: np.ndarray, idx: np.ndarray) -> np.ndarray:
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    k = _ARITY[kind]
    assert idx.ndim == 2 and idx.shape[1] == k
    out = np.zeros(idx.shape[0], dtype=np.int8)
    nq = idx.shape[0]
    if kind in ("in_sphere", "in_sphere_unperturbed"):
        getattr(lib, prefix + "in_sphere")(_ptr(pts), _ptr(idx), nq, int(kind == "in_sphere"), _ptr(out))
    elif kind in ("coplanar_in_circle", "coplanar_in_circle_unperturbed"):
        getattr(lib, prefix + "coplanar_in_circle")(_ptr(pts), _ptr(idx), nq,
                                                    int(kind == "coplanar_in_circle"), _ptr(out))
    else:
        getattr(lib, prefix + kind)(_ptr(pts), _ptr(idx), nq, _ptr(out))
    return out


def orc_predicate(kind: str, pts: np.ndarray, idx: np.ndarray) -> np.ndarray:
    return _pred(orc(), "orc_", kind, pts, idx)


def ref_predicate(kind: str, pts: np.ndarray, idx: np.ndarray) -> np.ndarray:
    return _pred(ref(), "ref_", kind, pts, idx)


def exact_predicate(kind: str, pts: np.ndarray, idx: np.ndarray) -> np.ndarray:
    return _pred(ref(), "exact_", kind, pts, idx)


def orc_spatial_sort(pts: np.ndarray) -> np.ndarray:
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    out = np.zeros(pts.shape[0], dtype=np.int32)
    orc().orc_spatial_sort(_ptr(pts), pts.shape[0], _ptr(out))
    return out


def orc_shuffle(n: int) -> np.ndarray:
    out = np.zeros(n, dtype=np.int32)
    orc().orc_shuffle(n, _ptr(out))
    return out


def ref_spatial_sort(pts: np.ndarray) -> np.ndarray:
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    out = np.zeros(pts.shape[0], dtype=np.int32)
    ref().ref_spatial_sort(_ptr(pts), pts.shape[0], _ptr(out))
    return out


def orc_build(pts: np.ndarray) -> dict:
    """Canonical cells (and all cells) of our CPU restatement."""
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    lib = orc()
    h = lib.orc_build(_ptr(pts), pts.shape[0])
    if not h:
        raise ValueError("non-finite input")
    try:
        nc, na = lib.orc_build_ncells(h), lib.orc_build_nall(h)
        cells = np.zeros((nc, 4), dtype=np.int32)
        allc = np.zeros((na, 4), dtype=np.int32)
        if nc:
            lib.orc_build_cells(h, _ptr(cells))
        if na:
            lib.orc_build_all(h, _ptr(allc))
        return {"cells": cells, "all": allc, "n_vertices": lib.orc_build_nvertices(h)}
    finally:
        lib.orc_build_free(h)


def ref_circumcenters(pts: np.ndarray, tets: np.ndarray, lazy: bool = False) -> np.ndarray:
    """The reference's del3d::circumcenter (or circumcenter_lazy) per tet
    (src/triangulation.cpp:805-930), (n, 3) float64."""
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    t = np.ascontiguousarray(tets, dtype=np.int32).reshape(-1, 4)
    out = np.zeros((t.shape[0], 3), dtype=np.float64)
    if t.shape[0]:
        ref().ref_circumcenter(_ptr(pts), _ptr(t), t.shape[0], int(lazy), _ptr(out))
    return out


def ref_build(pts: np.ndarray) -> dict:
    """The reference build's outputs, in the reference's own (allocation) order."""
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    lib = ref()
    h = lib.ref_build(_ptr(pts), pts.shape[0])
    try:
        nc, na = lib.ref_build_ncells(h), lib.ref_build_nall(h)
        cells = np.zeros((nc, 4), dtype=np.int32)
        allc = np.zeros((na, 4), dtype=np.int32)
        if nc:
            lib.ref_build_cells(h, _ptr(cells))
        if na:
            lib.ref_build_all(h, _ptr(allc))
        ninc = lib.ref_build_incident(h, None, None)
        offs = np.zeros(pts.shape[0] + 1, dtype=np.int64)
        data = np.zeros(max(ninc, 1), dtype=np.int32)
        lib.ref_build_incident(h, _ptr(offs), _ptr(data))
        return {"cells": cells, "all": allc, "n_vertices": lib.ref_build_nvertices(h),
                "incident_offsets": offs, "incident": data[:ninc]}
    finally:
        lib.ref_build_free(h)


def canonical_rotate(tets: np.ndarray) -> np.ndarray:
    t = np.ascontiguousarray(tets, dtype=np.int32).copy()
    if t.shape[0]:
        orc().orc_canonical_rotate(_ptr(t), t.shape[0])
    return t


def canonical_cells(tets: np.ndarray) -> np.ndarray:
    """Even rotation per tet, then lexicographic sort of the tets."""
    t = canonical_rotate(tets)
    if t.shape[0] == 0:
        return t.reshape(0, 4)
    order = np.lexsort((t[:, 3], t[:, 2], t[:, 1], t[:, 0]))
    return t[order]


def fnv1a_order(order: np.ndarray) -> int:
    """The reference's spatial-sort hash (4 low bytes of each index), tests/test_spatial_sort.cpp:46-51."""
    h = 1469598103934665603
    for v in np.asarray(order, dtype=np.int64).tolist():
        v &= 0xFFFFFFFFFFFFFFFF
        for b in range(4):
            h ^= (v >> (8 * b)) & 0xFF
            h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def fnv1a_cells(cells: np.ndarray) -> int:
    """The reference's cell-sequence hash, tests/test_delaunay.cpp:44-56."""
    h = 1469598103934665603

    def mix(v: int) -> None:
        nonlocal h
        v &= 0xFFFFFFFFFFFFFFFF
        for b in range(8):
            h ^= (v >> (8 * b)) & 0xFF
            h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF

    c = np.asarray(cells, dtype=np.int64).reshape(-1, 4)
    mix(c.shape[0])
    for v in c.ravel().tolist():
        mix(v)
    return h


# ---- the reference's test point sets -------------------------------------------

def _ps(fn, *args) -> np.ndarray:
    n = fn(*args, None)
    out = np.zeros((n, 3), dtype=np.float64)
    if n:
        fn(*args, _ptr(out))
    return out


def ps_cylinder(n: int, q: int = 32, seed: int = 1) -> np.ndarray:
    return _ps(ref().ps_cylinder, n, q, seed)


def ps_sphere(n: int, q: int = 32, seed: int = 2) -> np.ndarray:
    return _ps(ref().ps_sphere, n, q, seed)


def ps_torus(n: int, q: int = 32, seed: int = 3) -> np.ndarray:
    return _ps(ref().ps_torus, n, q, seed)


def ps_box_shell(m: int) -> np.ndarray:
    return _ps(ref().ps_box_shell, m)


def ps_lattice(nx: int, ny: int, nz: int) -> np.ndarray:
    return _ps(ref().ps_lattice, nx, ny, nz)


def ps_random_cube(n: int, seed: int = 4) -> np.ndarray:
    return _ps(ref().ps_random_cube, n, seed)


def ps_rng_below(seed: int, m: int, count: int) -> np.ndarray:
    out = np.zeros(count, dtype=np.int64)
    ref().ps_rng_below(seed, m, count, _ptr(out))
    return out


# ---- the benchmarks' synthetic point sets, without the product library ------------
#
# The same generators as del3d_b200.gen_set / mixed_workload (liboracle.so is
# compiled with del3d_b200/csrc/pointgen.cpp), so that the reference's timed arm
# of bench.py builds exactly the GPU arm's inputs without loading
# libdel3d_b200.so.  tests/test_oracle.py checks the two agree bit for bit.

DISTRIBUTIONS = ("uniform", "clusters", "lattice", "sphere")


def gen_set(dist: str, n: int, seed: int) -> np.ndarray:
    lib = orc()
    out = np.zeros((n, 3), dtype=np.float64)
    if n == 0:
        return out
    if dist == "uniform":
        lib.d3g_gen_uniform(n, seed, 0.0, 1.0, _ptr(out))
    elif dist == "clusters":
        lib.d3g_gen_clusters(n, seed, 8, 0.02, _ptr(out))
    elif dist == "lattice":
        lib.d3g_gen_lattice(n, _ptr(out))
    else:
        lib.d3g_gen_sphere(n, seed, 1.0, 1024, _ptr(out))
        _, first = np.unique(out, axis=0, return_index=True)
        out = out[np.sort(first)]
    return out


def gen_uniform(n: int, seed: int, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
    out = np.zeros((n, 3), dtype=np.float64)
    if n:
        orc().d3g_gen_uniform(n, seed, lo, hi, _ptr(out))
    return out


def mixed_workload(n_sets: int, lo: int = 32, hi: int = 65536, seed: int = 2024, first_seed: int = 1000):
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), n_sets))).astype(np.int64)
    dists = rng.integers(0, len(DISTRIBUTIONS), n_sets)
    return [gen_set(DISTRIBUTIONS[d], int(n), first_seed + k) for k, (n, d) in enumerate(zip(sizes, dists))]


# ---- the reference viewer's mesh reader ------------------------------------------------


class _RefMesh(ctypes.Structure):
    _fields_ = [("v", ctypes.POINTER(ctypes.c_double)), ("f", ctypes.POINTER(ctypes.c_int32)),
                ("nv", _I64), ("nf", _I64), ("err", ctypes.c_char * 512)]


def ref_meshio_available() -> bool:
    """Built, and linked against the shared C++ runtime (a copy of libstdc++
    linked in statically breaks its streams in a process that loaded the shared
    one, as numpy does)."""
    if not os.path.exists(_MESHIO_PATH):
        return False
    with open(_MESHIO_PATH, "rb") as fh:
        return b"libstdc++.so.6" in fh.read()


def _meshio_lib() -> ctypes.CDLL:
    global _meshio
    if _meshio is None:
        lib = ctypes.CDLL(_MESHIO_PATH)
        lib.ref_mesh_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(_RefMesh)]
        lib.ref_mesh_load.restype = _INT
        lib.ref_mesh_weld.argtypes = [_P, _I64, _P, _I64, ctypes.POINTER(_RefMesh)]
        lib.ref_mesh_weld.restype = None
        lib.ref_mesh_drop_non_finite.argtypes = [_P, _I64, _P, _I64, ctypes.POINTER(_RefMesh)]
        lib.ref_mesh_drop_non_finite.restype = _I64
        lib.ref_mesh_free.argtypes = [ctypes.POINTER(_RefMesh)]
        lib.ref_mesh_formats.restype = ctypes.c_char_p
        lib.ref_mesh_error.restype = ctypes.c_char_p
        _meshio = lib
    return _meshio


def _ref_arrays(m: _RefMesh):
    v = np.ctypeslib.as_array(m.v, shape=(int(m.nv) * 3,)).reshape(-1, 3).copy() if m.nv \
        else np.zeros((0, 3), dtype=np.float64)
    f = np.ctypeslib.as_array(m.f, shape=(int(m.nf) * 3,)).reshape(-1, 3).copy() if m.nf \
        else np.zeros((0, 3), dtype=np.int32)
    return v, f


def ref_mesh_load(path, with_status=False):
    """meshio::load of the reference: (vertices, faces, error text or "").  The
    text is decoded with surrogateescape (it may quote bytes of the file).  With
    `with_status`, also 2 when the reference threw (it would abort a program)."""
    lib = _meshio_lib()
    m = _RefMesh()
    rc = lib.ref_mesh_load(os.fsencode(path), ctypes.byref(m))
    try:
        v, f = _ref_arrays(m)
        err = lib.ref_mesh_error().decode(errors="surrogateescape")
        return (v, f, err, rc) if with_status else (v, f, err)
    finally:
        lib.ref_mesh_free(ctypes.byref(m))


def ref_weld(v, f):
    """meshio::weld of the reference: (vertices, faces)."""
    lib = _meshio_lib()
    v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
    f = np.ascontiguousarray(f, dtype=np.int32).reshape(-1, 3)
    m = _RefMesh()
    lib.ref_mesh_weld(_ptr(v), v.shape[0], _ptr(f), f.shape[0], ctypes.byref(m))
    try:
        return _ref_arrays(m)
    finally:
        lib.ref_mesh_free(ctypes.byref(m))


def ref_drop_non_finite(v, f):
    """meshio::drop_non_finite of the reference: (vertices, faces, dropped)."""
    lib = _meshio_lib()
    v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
    f = np.ascontiguousarray(f, dtype=np.int32).reshape(-1, 3)
    m = _RefMesh()
    d = lib.ref_mesh_drop_non_finite(_ptr(v), v.shape[0], _ptr(f), f.shape[0], ctypes.byref(m))
    try:
        vv, ff = _ref_arrays(m)
        return vv, ff, int(d)
    finally:
        lib.ref_mesh_free(ctypes.byref(m))


def ref_mesh_formats() -> str:
    return _meshio_lib().ref_mesh_formats().decode()
