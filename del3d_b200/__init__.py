"""del3d_b200 - del3d's Delaunay::build hot path on B200 (sm_100a).

Python host side over the C ABI of ``libdel3d_b200.so`` (``include/del3d_b200.h``).
It mirrors the reference's public interface (``include/del3d/delaunay.h``,
``predicates.h``, ``predicates2.h``, ``spatial_sort.h`` in the del3d tree):

* :class:`Delaunay` - ``build(points)``, ``finite_cells()``, ``all_cells()``,
  ``incident_cells()``, ``number_of_vertices()``;
* :func:`orient3d`, :func:`in_sphere`, :func:`in_sphere_unperturbed`,
  :func:`orient2d`, :func:`coplanar_orientation`, :func:`coplanar_in_circle`,
  :func:`coplanar_in_circle_unperturbed`, :func:`collinear` - batched over index
  tuples into one point table;
* :func:`spatial_sort` - the reference insertion order, bit for bit;
* :func:`load_mesh`, :func:`weld`, :func:`drop_non_finite`, :func:`read_xyz`,
  :func:`load_point_sets` - the reference viewer's input readers, on the host.

Everything but the input readers runs on the GPU; there is no CPU fallback.  Importing works without a
GPU (the library loads), but every call then fails with :class:`Del3dError`.

One documented difference: ``finite_cells()`` comes back in a canonical order
(each tet rotated by an even permutation so its smallest index leads, tets
sorted lexicographically) instead of the reference's cell-allocation order; the
set of tets is the reference's.
"""
from __future__ import annotations

import ctypes
import os
from typing import List, Optional, Sequence

import numpy as np

__all__ = [
    "Del3dError", "Delaunay", "Point3", "orient3d", "in_sphere", "in_sphere_unperturbed",
    "orient2d", "coplanar_orientation", "coplanar_in_circle", "coplanar_in_circle_unperturbed",
    "collinear", "spatial_sort", "library", "LIB_PATH", "predicate_stats", "circumcenters",
    "circumcenter", "circumcenter_lazy", "Server", "Request", "pool_usage",
    "release_cached_memory", "load_mesh", "read_xyz", "weld", "drop_non_finite",
    "supported_formats", "load_point_sets", "partition_sets", "validate_cells",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdel3d_b200.so")

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I32 = ctypes.c_int32
_INT = ctypes.c_int


# d3g_status values (include/del3d_b200.h).
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_INVALID_INPUT = 2
ERR_OOM = 3
ERR_EXACT_CAPACITY = 4
ERR_CAVITY_CAPACITY = 5
ERR_WALK_LIMIT = 6
ERR_ROUND_LIMIT = 7
ERR_CUDA = 8
ERR_INTERNAL = 9
ERR_NO_DEVICE = 10
ERR_NOT_READY = 11


class Del3dError(RuntimeError):
    """A non-OK status from the C ABI (the reference has no error channel; this
    library never fails silently)."""

    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        msg = f"{where}: {_status_string(status)}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


class BuildStats(ctypes.Structure):
    """What a build did (d3g_build_stats)."""
    _fields_ = [("rounds", _I32), ("attempts", _I64), ("region_tets", _I64),
                ("boundary_facets", _I64), ("ms_order", ctypes.c_double),
                ("ms_rounds", ctypes.c_double), ("ms_output", ctypes.c_double),
                ("ms_cavity", ctypes.c_double), ("ms_check", ctypes.c_double),
                ("ms_restar", ctypes.c_double), ("launches_cavity", _I64),
                ("walk_steps", _I64), ("bfs_steps", _I64), ("ms_async", ctypes.c_double),
                ("launches_async", _I64), ("async_inserted", _I64), ("conflict_tests", _I64),
                ("uncertain_tests", _I64), ("tie_breaks", _I64), ("max_region_tets", _I64),
                ("deferred_points", _I64)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class _Result(ctypes.Structure):
    _fields_ = [
        ("n_points", _I64), ("n_vertices", _I64), ("n_cells", _I64),
        ("cells", ctypes.POINTER(_I32)), ("n_all", _I64), ("all_cells", ctypes.POINTER(_I32)),
        ("incident_offsets", ctypes.POINTER(_I64)), ("incident", ctypes.POINTER(_I32)),
        ("device_ms", ctypes.c_double), ("stats", BuildStats),
    ]


class _Options(ctypes.Structure):
    _fields_ = [("want_all_cells", _I32), ("want_incident", _I32), ("chunk", _I32),
                ("max_rounds", _I32), ("timing", _I32), ("alpha_small", _I32), ("split", _I32),
                ("lanes", _I32), ("schedule", _I32), ("tet_capacity", _I32), ("walk_limit", _I32),
                ("cavity_capacity", _I32), ("validate", _I32), ("level_growth", _I32)]


class _BatchResult(ctypes.Structure):
    _fields_ = [("n_sets", _I32), ("cell_offsets", ctypes.POINTER(_I64)),
                ("cells", ctypes.POINTER(_I32)), ("n_vertices", ctypes.POINTER(_I64)),
                ("device_ms", ctypes.c_double), ("stats", BuildStats)]


class _ServerOptions(ctypes.Structure):
    _fields_ = [("slots", _I32), ("hbm_budget_bytes", _I64), ("max_batch_sets", _I32),
                ("max_batch_points", _I64), ("device", _I32)]


class _RequestResult(ctypes.Structure):
    _fields_ = [("status", _I32), ("n_points", _I64), ("n_vertices", _I64), ("n_cells", _I64),
                ("cells", ctypes.POINTER(_I32)), ("t_submit", ctypes.c_double),
                ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double), ("batch_sets", _I32)]


class _ServerStats(ctypes.Structure):
    _fields_ = [("submitted", _I64), ("completed", _I64), ("queued", _I64), ("batches", _I64),
                ("batched_requests", _I64), ("bytes_in_use", _I64), ("peak_bytes_in_use", _I64),
                ("hbm_budget_bytes", _I64), ("peak_in_flight_requests", _I64), ("slots", _I32)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class _Tuning(ctypes.Structure):
    _fields_ = [("schedule", _I32), ("chunk", _I32), ("alpha_small", _I32), ("lanes", _I32),
                ("ms", ctypes.c_double), ("candidates", _I32)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class _PredStats(ctypes.Structure):
    _fields_ = [("n_queries", _I64), ("n_exact", _I64)]


class _Mesh(ctypes.Structure):
    _fields_ = [("vertices", ctypes.POINTER(ctypes.c_double)), ("faces", ctypes.POINTER(_I32)),
                ("n_vertices", _I64), ("n_faces", _I64)]


class _PointSets(ctypes.Structure):
    _fields_ = [("xyz", ctypes.POINTER(ctypes.c_double)), ("set_offsets", ctypes.POINTER(_I64)),
                ("dropped", ctypes.POINTER(_I64)), ("n_sets", _INT)]


_lib: Optional[ctypes.CDLL] = None


def library() -> ctypes.CDLL:
    """The loaded C library.  Raises if it was not built (``python -c
    'import __graft_entry__ as g; g.build()'``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"del3d_b200: {LIB_PATH} is missing; build it with __graft_entry__.build()")
    lib = ctypes.CDLL(LIB_PATH)
    lib.d3g_status_string.argtypes = [_INT]
    lib.d3g_status_string.restype = ctypes.c_char_p
    lib.d3g_last_error.argtypes = []
    lib.d3g_last_error.restype = ctypes.c_char_p
    lib.d3g_predicate_arity.argtypes = [_INT]
    lib.d3g_predicate_arity.restype = _INT
    lib.d3g_predicates.argtypes = [_P, _I64, _P, _I64, _INT, _P, ctypes.POINTER(_PredStats)]
    lib.d3g_predicates_device.argtypes = [_P, _I64, _P, _I64, _INT, _P, _P, ctypes.POINTER(_PredStats)]
    lib.d3g_orient2d.argtypes = [_P, _I64, _P]
    lib.d3g_spatial_sort.argtypes = [_P, _I64, _P]
    lib.d3g_spatial_sort_device.argtypes = [_P, _I64, _P, _P]
    lib.d3g_shuffle_device.argtypes = [_I64, _P, _P]
    lib.d3g_options_default.argtypes = [ctypes.POINTER(_Options)]
    lib.d3g_release_cached_memory.argtypes = []
    lib.d3g_release_cached_memory.restype = _INT
    lib.d3g_build.argtypes = [_P, _I64, ctypes.POINTER(_Options), ctypes.POINTER(_Result)]
    lib.d3g_result_free.argtypes = [ctypes.POINTER(_Result)]
    lib.d3g_build_device.argtypes = [_P, _I64, ctypes.POINTER(_Options), _P, _I64,
                                     ctypes.POINTER(_I64), ctypes.POINTER(_I64), _P,
                                     ctypes.POINTER(BuildStats)]
    lib.d3g_build_batch.argtypes = [_P, _P, _I32, ctypes.POINTER(_Options), ctypes.POINTER(_BatchResult)]
    lib.d3g_build_batch.restype = _INT
    lib.d3g_batch_result_free.argtypes = [ctypes.POINTER(_BatchResult)]
    lib.d3g_build_batch_device.argtypes = [_P, _P, _I32, ctypes.POINTER(_Options), _P, _I64, _P, _P, _P,
                                           ctypes.POINTER(BuildStats)]
    lib.d3g_build_batch_device.restype = _INT
    lib.d3g_circumcenters.argtypes = [_P, _I64, _P, _I64, _INT, _P, ctypes.POINTER(_PredStats)]
    lib.d3g_circumcenters.restype = _INT
    lib.d3g_circumcenters_device.argtypes = [_P, _I64, _P, _I64, _INT, _P, _P, ctypes.POINTER(_PredStats)]
    lib.d3g_circumcenters_device.restype = _INT
    lib.d3g_server_options_default.argtypes = [ctypes.POINTER(_ServerOptions)]
    lib.d3g_server_options_default.restype = None
    lib.d3g_server_create.argtypes = [ctypes.POINTER(_ServerOptions), ctypes.POINTER(_P)]
    lib.d3g_server_create.restype = _INT
    lib.d3g_server_submit.argtypes = [_P, _P, _I64, ctypes.POINTER(_I64)]
    lib.d3g_server_submit.restype = _INT
    lib.d3g_server_wait.argtypes = [_P, _I64, ctypes.c_double, ctypes.POINTER(_RequestResult)]
    lib.d3g_server_wait.restype = _INT
    lib.d3g_request_result_free.argtypes = [ctypes.POINTER(_RequestResult)]
    lib.d3g_request_result_free.restype = None
    lib.d3g_server_get_stats.argtypes = [_P, ctypes.POINTER(_ServerStats)]
    lib.d3g_server_get_stats.restype = _INT
    lib.d3g_server_destroy.argtypes = [_P]
    lib.d3g_server_destroy.restype = _INT
    lib.d3g_microbench_fp64.argtypes = [_I64, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), _P]
    lib.d3g_microbench_fp64.restype = _INT
    lib.d3g_autotune_device.argtypes = [_P, _P, _I32, _P, ctypes.POINTER(_Tuning)]
    lib.d3g_autotune_device.restype = _INT
    lib.d3g_get_tuning.argtypes = [ctypes.POINTER(_Tuning)]
    lib.d3g_get_tuning.restype = _INT
    lib.d3g_reset_tuning.argtypes = []
    lib.d3g_reset_tuning.restype = _INT
    lib.d3g_pool_usage.argtypes = [ctypes.POINTER(_I64), ctypes.POINTER(_I64), _INT]
    lib.d3g_pool_usage.restype = _INT
    lib.d3g_gen_uniform.argtypes = [_I64, ctypes.c_uint32, ctypes.c_double, ctypes.c_double, _P]
    lib.d3g_gen_sphere.argtypes = [_I64, ctypes.c_uint32, ctypes.c_double, _I32, _P]
    lib.d3g_gen_clusters.argtypes = [_I64, ctypes.c_uint32, _I32, ctypes.c_double, _P]
    lib.d3g_gen_lattice.argtypes = [_I64, _P]
    for name in ("d3g_mesh_load", "d3g_read_xyz"):
        getattr(lib, name).argtypes = [ctypes.c_char_p, ctypes.POINTER(_Mesh)]
        getattr(lib, name).restype = _INT
    lib.d3g_mesh_weld.argtypes = [ctypes.POINTER(_Mesh)]
    lib.d3g_mesh_weld.restype = _INT
    lib.d3g_mesh_drop_non_finite.argtypes = [ctypes.POINTER(_Mesh), ctypes.POINTER(_I64)]
    lib.d3g_mesh_drop_non_finite.restype = _INT
    lib.d3g_mesh_free.argtypes = [ctypes.POINTER(_Mesh)]
    lib.d3g_mesh_free.restype = None
    lib.d3g_mesh_supported_formats.argtypes = []
    lib.d3g_mesh_supported_formats.restype = ctypes.c_char_p
    lib.d3g_load_point_sets.argtypes = [ctypes.POINTER(ctypes.c_char_p), _INT, _INT, ctypes.POINTER(_PointSets)]
    lib.d3g_load_point_sets.restype = _INT
    lib.d3g_point_sets_free.argtypes = [ctypes.POINTER(_PointSets)]
    lib.d3g_point_sets_free.restype = None
    lib.d3g_validate_cells.argtypes = [_P, _I64, _I64]
    lib.d3g_validate_cells.restype = _INT
    for name in ("d3g_predicates", "d3g_predicates_device", "d3g_orient2d", "d3g_spatial_sort",
                 "d3g_spatial_sort_device", "d3g_shuffle_device", "d3g_build", "d3g_build_device"):
        getattr(lib, name).restype = _INT
    _lib = lib
    return lib


def _status_string(status: int) -> str:
    try:
        return library().d3g_status_string(status).decode()
    except ImportError:
        return f"status {status}"


def _check(status: int, where: str) -> None:
    if status != 0:
        detail = library().d3g_last_error().decode(errors="replace")   # may quote file bytes
        raise Del3dError(status, where, detail)


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _points(points) -> np.ndarray:
    """(n, 3) float64 C-contiguous view/copy of `points` (array-like or Point3 list)."""
    if isinstance(points, np.ndarray):
        a = points
    elif len(points) and hasattr(points[0], "x"):
        a = np.array([(p.x, p.y, p.z) for p in points], dtype=np.float64)
    else:
        a = np.asarray(points, dtype=np.float64)
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1, 3)
    return a


class Point3:
    """A point (reference ``include/del3d/spatial_sort.h:31``)."""

    __slots__ = ("x", "y", "z")

    def __init__(self, x: float, y: float, z: float):
        self.x, self.y, self.z = float(x), float(y), float(z)

    def __iter__(self):
        yield self.x
        yield self.y
        yield self.z

    def __repr__(self) -> str:
        return f"Point3({self.x!r}, {self.y!r}, {self.z!r})"


# ---- predicates -----------------------------------------------------------------

ORIENT3D, IN_SPHERE, IN_SPHERE_UNPERTURBED = 0, 1, 2
COPLANAR_ORIENTATION3, COPLANAR_ORIENTATION4 = 3, 4
COPLANAR_IN_CIRCLE, COPLANAR_IN_CIRCLE_UNPERTURBED, COLLINEAR = 5, 6, 7

_last_pred_stats = (0, 0)


def predicate_stats():
    """(queries, queries that reached the exact stage) of the last predicate call."""
    return _last_pred_stats


def _predicate(kind: int, points, idx) -> np.ndarray:
    global _last_pred_stats
    lib = library()
    pts = _points(points)
    k = lib.d3g_predicate_arity(kind)
    ix = np.ascontiguousarray(idx, dtype=np.int32).reshape(-1, k)
    if kind == ORIENT3D and ix.ctypes.data % 16:
        ix = np.array(ix, dtype=np.int32, copy=True, order="C")
    out = np.zeros(ix.shape[0], dtype=np.int8)
    st = _PredStats()
    _check(lib.d3g_predicates(_ptr(pts), pts.shape[0], _ptr(ix), ix.shape[0], kind, _ptr(out),
                              ctypes.byref(st)), "predicates")
    _last_pred_stats = (st.n_queries, st.n_exact)
    return out


def orient3d(points, idx) -> np.ndarray:
    """Sign of |b-a, c-a, d-a| per row (a, b, c, d) of `idx` (reference predicates.h:28)."""
    return _predicate(ORIENT3D, points, idx)


def in_sphere(points, idx) -> np.ndarray:
    """Perturbed in-sphere per row (a, b, c, d, e); never 0 (reference predicates.h:52)."""
    return _predicate(IN_SPHERE, points, idx)


def in_sphere_unperturbed(points, idx) -> np.ndarray:
    """Raw in-sphere per row; 0 when cospherical (reference predicates.h:57)."""
    return _predicate(IN_SPHERE_UNPERTURBED, points, idx)


def coplanar_orientation(points, idx) -> np.ndarray:
    """Rows of 3 (p,q,r) or 4 (p,q,r,s) indices (reference predicates2.h:33,40)."""
    ix = np.asarray(idx)
    kind = COPLANAR_ORIENTATION3 if ix.reshape(ix.shape[0], -1).shape[1] == 3 else COPLANAR_ORIENTATION4
    return _predicate(kind, points, ix)


def coplanar_in_circle(points, idx) -> np.ndarray:
    """Perturbed in-circle per row (p0, p1, p2, p) (reference predicates2.h:66)."""
    return _predicate(COPLANAR_IN_CIRCLE, points, idx)


def coplanar_in_circle_unperturbed(points, idx) -> np.ndarray:
    """Raw in-circle per row (reference predicates2.h:70)."""
    return _predicate(COPLANAR_IN_CIRCLE_UNPERTURBED, points, idx)


def collinear(points, idx) -> np.ndarray:
    """1 where the row (p, q, r) is exactly collinear (reference predicates2.h:46)."""
    return _predicate(COLLINEAR, points, idx)


def orient2d(six) -> np.ndarray:
    """Sign of |q-p, r-p| per row (px, py, qx, qy, rx, ry) (reference predicates2.h:27)."""
    lib = library()
    a = np.ascontiguousarray(six, dtype=np.float64).reshape(-1, 6)
    out = np.zeros(a.shape[0], dtype=np.int8)
    _check(lib.d3g_orient2d(_ptr(a), a.shape[0], _ptr(out)), "orient2d")
    return out


def circumcenters(points, tets, lazy: bool = False) -> np.ndarray:
    """Circumcentre of every tet (rows of 4 indices into `points`), (n, 3)
    float64: del3d::circumcenter, or del3d::circumcenter_lazy with lazy=True
    (reference delaunay.h:29, :48).  A coplanar tet gives its first vertex."""
    global _last_pred_stats
    lib = library()
    pts = _points(points)
    t = np.ascontiguousarray(tets, dtype=np.int32).reshape(-1, 4)
    out = np.zeros((t.shape[0], 3), dtype=np.float64)
    st = _PredStats()
    _check(lib.d3g_circumcenters(_ptr(pts), pts.shape[0], _ptr(t), t.shape[0], int(lazy), _ptr(out),
                                 ctypes.byref(st)), "circumcenters")
    _last_pred_stats = (st.n_queries, st.n_exact)
    return out


def circumcenter(p0, p1, p2, p3) -> Point3:
    """del3d::circumcenter of one tetrahedron (reference delaunay.h:29)."""
    c = circumcenters([tuple(p0), tuple(p1), tuple(p2), tuple(p3)], [[0, 1, 2, 3]])[0]
    return Point3(*c)


def circumcenter_lazy(p, q, r, s) -> Point3:
    """del3d::circumcenter_lazy of one tetrahedron (reference delaunay.h:48)."""
    c = circumcenters([tuple(p), tuple(q), tuple(r), tuple(s)], [[0, 1, 2, 3]], lazy=True)[0]
    return Point3(*c)


def spatial_sort(points, order: Optional[List[int]] = None) -> np.ndarray:
    """The reference insertion order of `points` (reference spatial_sort.h:37).

    As in the reference, `order` (if given) must be 0..n-1 on entry; it is
    reordered in place when it is a list, and the order is also returned."""
    lib = library()
    pts = _points(points)
    out = np.zeros(pts.shape[0], dtype=np.int32)
    if pts.shape[0]:
        _check(lib.d3g_spatial_sort(_ptr(pts), pts.shape[0], _ptr(out)), "spatial_sort")
    if order is not None:
        order[:] = out.tolist()
    return out


# ---- the build ------------------------------------------------------------------


class Delaunay:
    """The Delaunay triangulation of a point set (reference delaunay.h:62-92),
    built on the GPU."""

    def __init__(self) -> None:
        self._cells = np.zeros((0, 4), dtype=np.int32)
        self._all = np.zeros((0, 4), dtype=np.int32)
        self._inc_off = np.zeros(1, dtype=np.int64)
        self._inc = np.zeros(0, dtype=np.int32)
        self._n_vertices = 0
        self.rounds = 0
        self.device_ms = 0.0
        self.stats = {}

    def build(self, points, chunk: int = 0, all_cells: bool = True, incident: bool = True) -> None:
        """Builds the triangulation.  Points equal to an earlier point are
        ignored; a repeated point is reported under the index of its copy that
        comes last in the spatial-sort order, as in the reference."""
        lib = library()
        pts = _points(points)
        opts = _Options()
        lib.d3g_options_default(ctypes.byref(opts))
        if chunk:
            opts.chunk = int(chunk)
        opts.want_all_cells = int(all_cells)
        opts.want_incident = int(incident)
        res = _Result()
        _check(lib.d3g_build(_ptr(pts), pts.shape[0], ctypes.byref(opts), ctypes.byref(res)), "build")
        try:
            nc, na = res.n_cells, res.n_all
            self._cells = (np.ctypeslib.as_array(res.cells, shape=(nc * 4,)).reshape(nc, 4).copy()
                           if nc else np.zeros((0, 4), dtype=np.int32))
            self._all = (np.ctypeslib.as_array(res.all_cells, shape=(na * 4,)).reshape(na, 4).copy()
                         if na else np.zeros((0, 4), dtype=np.int32))
            n = pts.shape[0]
            if res.incident_offsets:
                self._inc_off = np.ctypeslib.as_array(res.incident_offsets, shape=(n + 1,)).copy()
            else:                                   # incident lists not asked for
                self._inc_off = np.zeros(n + 1, dtype=np.int64)
            ninc = int(self._inc_off[-1])
            self._inc = (np.ctypeslib.as_array(res.incident, shape=(ninc,)).copy()
                         if ninc else np.zeros(0, dtype=np.int32))
            self._n_vertices = int(res.n_vertices)
            self.stats = res.stats.as_dict()
            self.rounds = int(res.stats.rounds)
            self.device_ms = float(res.device_ms)
        finally:
            lib.d3g_result_free(ctypes.byref(res))

    def finite_cells(self) -> np.ndarray:
        """(n_cells, 4) int32 finite tets, canonical order."""
        return self._cells

    def all_cells(self) -> np.ndarray:
        """Every tet, infinite ones included (-1 = the infinite vertex), canonical order."""
        return self._all

    def incident_cells(self) -> List[np.ndarray]:
        """Per input point, the ascending indices into finite_cells() of its cells."""
        o = self._inc_off
        return [self._inc[o[i]:o[i + 1]] for i in range(len(o) - 1)]

    def incident_csr(self):
        """incident_cells() as CSR arrays (offsets[n+1], indices)."""
        return self._inc_off, self._inc

    def number_of_vertices(self) -> int:
        return self._n_vertices


def _apply(opts, **kw):
    """Sets the options given (not None); the rest keep d3g_options_default's
    values (which an autotuning run may have chosen)."""
    for name, value in kw.items():
        if value is not None:
            setattr(opts, name, int(value))


def build_device(points_dev, out=None, stream: int = 0, chunk: Optional[int] = None, timing: bool = False,
                 stats: Optional[dict] = None, alpha_small: Optional[int] = None, split: Optional[int] = None,
                 lanes: Optional[int] = None, schedule: Optional[int] = None, max_rounds: Optional[int] = None,
                 tet_capacity: Optional[int] = None, walk_limit: Optional[int] = None,
                 cavity_capacity: Optional[int] = None, validate: Optional[bool] = None,
                 level_growth: Optional[int] = None):
    """Builds from a device-resident torch tensor (n, 3) float64 on `stream`
    (a raw cudaStream_t handle; 0 = default) and returns the canonical finite
    cells as a device int32 tensor view (n_cells, 4) and the vertex count.
    `out` may supply the (cap, 4) int32 output buffer.  Synchronises `stream`.
    max_rounds / tet_capacity / walk_limit / cavity_capacity lower the build's
    limits (d3g_options), which makes their failure statuses reachable;
    `validate` checks the device tet table's invariants after every level."""
    import torch

    lib = library()
    assert points_dev.is_cuda and points_dev.dtype == torch.float64
    x = points_dev.contiguous()
    n = x.shape[0]
    if out is None:
        out = torch.empty((8 * n + 64, 4), dtype=torch.int32, device=x.device)
    nc, nv = _I64(0), _I64(0)
    opts = _Options()
    lib.d3g_options_default(ctypes.byref(opts))
    _apply(opts, chunk=chunk, timing=int(timing), alpha_small=alpha_small, split=split, lanes=lanes,
           schedule=schedule, max_rounds=max_rounds, tet_capacity=tet_capacity, walk_limit=walk_limit,
           cavity_capacity=cavity_capacity, validate=None if validate is None else int(validate),
           level_growth=level_growth)
    st = BuildStats()
    _check(lib.d3g_build_device(x.data_ptr(), n, ctypes.byref(opts), out.data_ptr(), out.shape[0],
                                ctypes.byref(nc), ctypes.byref(nv), _P(stream), ctypes.byref(st)),
           "build_device")
    if stats is not None:
        stats.update(st.as_dict())
    return out[: nc.value], nv.value


def build_batch(sets, chunk: int = 0, stats: Optional[dict] = None):
    """Builds many independent point sets in one call.  Returns, per set, its
    finite cells ((k, 4) int32, indices local to the set, canonical order - the
    same as Delaunay().build(set).finite_cells()) and its vertex count."""
    lib = library()
    arrays = [_points(a) for a in sets]
    if not arrays:
        return [], []
    offs = np.zeros(len(arrays) + 1, dtype=np.int64)
    offs[1:] = np.cumsum([a.shape[0] for a in arrays])
    xyz = np.ascontiguousarray(np.concatenate(arrays) if offs[-1] else np.zeros((1, 3)))
    opts = _Options()
    lib.d3g_options_default(ctypes.byref(opts))
    if chunk:
        opts.chunk = int(chunk)
    res = _BatchResult()
    _check(lib.d3g_build_batch(_ptr(xyz), _ptr(offs), len(arrays), ctypes.byref(opts), ctypes.byref(res)),
           "build_batch")
    try:
        co = np.ctypeslib.as_array(res.cell_offsets, shape=(len(arrays) + 1,)).copy()
        nv = np.ctypeslib.as_array(res.n_vertices, shape=(len(arrays),)).copy()
        total = int(co[-1])
        cells = (np.ctypeslib.as_array(res.cells, shape=(total * 4,)).reshape(total, 4).copy()
                 if total else np.zeros((0, 4), dtype=np.int32))
        if stats is not None:
            stats.update(res.stats.as_dict())
            stats["device_ms"] = res.device_ms
    finally:
        lib.d3g_batch_result_free(ctypes.byref(res))
    return [cells[co[i]:co[i + 1]] for i in range(len(arrays))], [int(v) for v in nv]


def build_batch_device(points_dev, set_offsets, out=None, stream: int = 0, chunk: Optional[int] = None,
                       stats: Optional[dict] = None, alpha_small: Optional[int] = None,
                       split: Optional[int] = None, lanes: Optional[int] = None,
                       schedule: Optional[int] = None, validate: Optional[bool] = None,
                       level_growth: Optional[int] = None):
    """Device-resident form of build_batch: `points_dev` (n, 3) float64 CUDA
    tensor holding the sets back to back, `set_offsets` (n_sets + 1) host
    int64.  Returns the device cells tensor (all sets), the cell offsets per
    set and the vertex counts per set.  Synchronises `stream`.  `validate`:
    check the device tet table's invariants after every level (debug)."""
    import torch

    lib = library()
    offs = np.ascontiguousarray(set_offsets, dtype=np.int64)
    nsets = offs.shape[0] - 1
    x = points_dev.contiguous()
    if out is None:
        out = torch.empty((8 * x.shape[0] + 64, 4), dtype=torch.int32, device=x.device)
    co = np.zeros(nsets + 1, dtype=np.int64)
    nv = np.zeros(nsets, dtype=np.int64)
    opts = _Options()
    lib.d3g_options_default(ctypes.byref(opts))
    _apply(opts, chunk=chunk, alpha_small=alpha_small, split=split, lanes=lanes, schedule=schedule,
           validate=None if validate is None else int(validate), level_growth=level_growth)
    st = BuildStats()
    _check(lib.d3g_build_batch_device(x.data_ptr(), _ptr(offs), nsets, ctypes.byref(opts), out.data_ptr(),
                                      out.shape[0], _ptr(co), _ptr(nv), _P(stream), ctypes.byref(st)),
           "build_batch_device")
    if stats is not None:
        stats.update(st.as_dict())
    return out[: int(co[-1])], co, nv


# ---- serving --------------------------------------------------------------------


NOT_READY = 11


class Request:
    """A completed request: its finite cells (canonical order, indices into the
    request's points), vertex count and timestamps (seconds since the server
    started)."""

    __slots__ = ("cells", "n_vertices", "t_submit", "t_admit", "t_done", "batch_sets")

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


class Server:
    """Continuous-batching request server on one GPU (d3g_server_*).

    ``submit(points)`` queues a triangulation request and returns a ticket;
    ``wait(ticket)`` returns its :class:`Request`.  Free slots (each a worker
    with its own CUDA stream) take the pending requests in arrival order while
    they fit the batch limits and the device-memory budget, so requests that
    arrive while others run are admitted as slots and memory free up.  Each
    request's cells equal ``Delaunay().build(points).finite_cells()``.
    Thread-safe; use as a context manager or call :meth:`close`."""

    def __init__(self, slots: int = 4, hbm_budget_bytes: int = 0, max_batch_sets: int = 1024,
                 max_batch_points: int = 8 << 20, device: int = -1):
        lib = library()
        o = _ServerOptions()
        lib.d3g_server_options_default(ctypes.byref(o))
        o.slots, o.hbm_budget_bytes = int(slots), int(hbm_budget_bytes)
        o.max_batch_sets, o.max_batch_points, o.device = int(max_batch_sets), int(max_batch_points), int(device)
        h = _P()
        _check(lib.d3g_server_create(ctypes.byref(o), ctypes.byref(h)), "server_create")
        self._h = h
        self._keep = {}          # ticket -> input array (borrowed by the server until done)

    def submit(self, points) -> int:
        pts = _points(points)
        t = _I64(0)
        _check(library().d3g_server_submit(self._h, _ptr(pts) if pts.shape[0] else None, pts.shape[0],
                                           ctypes.byref(t)), "server_submit")
        self._keep[t.value] = pts
        return t.value

    def wait(self, ticket: int, timeout: float = -1.0) -> Request:
        lib = library()
        res = _RequestResult()
        st = lib.d3g_server_wait(self._h, int(ticket), float(timeout), ctypes.byref(res))
        if st == NOT_READY:
            raise TimeoutError(f"request {ticket} not complete within {timeout} s")
        self._keep.pop(int(ticket), None)
        try:
            _check(st, "server_wait")
            r = Request()
            nc = res.n_cells
            r.cells = (np.ctypeslib.as_array(res.cells, shape=(nc * 4,)).reshape(nc, 4).copy()
                       if nc else np.zeros((0, 4), dtype=np.int32))
            r.n_vertices = int(res.n_vertices)
            r.t_submit, r.t_admit, r.t_done = res.t_submit, res.t_admit, res.t_done
            r.batch_sets = int(res.batch_sets)
            return r
        finally:
            lib.d3g_request_result_free(ctypes.byref(res))

    def stats(self) -> dict:
        st = _ServerStats()
        _check(library().d3g_server_get_stats(self._h, ctypes.byref(st)), "server_stats")
        return st.as_dict()

    def close(self) -> None:
        if getattr(self, "_h", None):
            library().d3g_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fp64_throughput(iters: int = 1 << 16, stream: int = 0):
    """(separate DADD/DMUL operations/s, DFMA/s) of the current device."""
    a, f = ctypes.c_double(0), ctypes.c_double(0)
    _check(library().d3g_microbench_fp64(int(iters), ctypes.byref(a), ctypes.byref(f), _P(stream)),
           "microbench_fp64")
    return a.value, f.value


def pool_usage(reset_high: bool = False):
    """(bytes in use, high-water mark) of the current device's stream-ordered
    pool; blocks the library keeps cached for later builds count as in use."""
    u, h = _I64(0), _I64(0)
    _check(library().d3g_pool_usage(ctypes.byref(u), ctypes.byref(h), int(reset_high)), "pool_usage")
    return u.value, h.value


def release_cached_memory() -> None:
    """Returns the cached device blocks and the pool's reserve to the CUDA driver and
    unpins the cached host result blocks (synchronises the device)."""
    _check(library().d3g_release_cached_memory(), "release_cached_memory")


# ---- autotuning ---------------------------------------------------------------------


def autotune(points_dev, set_offsets, stream: int = 0) -> dict:
    """Times builds of the sets `set_offsets` of the device tensor `points_dev`
    under the candidate speed settings and makes the fastest this device's
    default (d3g_autotune_device).  Returns the chosen setting."""
    offs = np.ascontiguousarray(set_offsets, dtype=np.int64)
    t = _Tuning()
    _check(library().d3g_autotune_device(points_dev.contiguous().data_ptr(), _ptr(offs), offs.shape[0] - 1,
                                         _P(stream), ctypes.byref(t)), "autotune")
    return t.as_dict()


def get_tuning() -> dict:
    t = _Tuning()
    _check(library().d3g_get_tuning(ctypes.byref(t)), "get_tuning")
    return t.as_dict()


def reset_tuning() -> None:
    _check(library().d3g_reset_tuning(), "reset_tuning")


# ---- synthetic inputs -------------------------------------------------------------


def gen_uniform(n: int, seed: int, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
    """n points uniform in [lo, hi)^3 from std::mt19937(seed), u01 = word * 2^-32."""
    out = np.zeros((n, 3), dtype=np.float64)
    if n:
        library().d3g_gen_uniform(n, seed, lo, hi, _ptr(out))
    return out


def gen_sphere(n: int, seed: int, r: float = 1.0, q: int = 1024, dedupe: bool = True) -> np.ndarray:
    """Sphere samples snapped to a 1/q grid (duplicates removed, first kept)."""
    out = np.zeros((n, 3), dtype=np.float64)
    if n:
        library().d3g_gen_sphere(n, seed, r, q, _ptr(out))
    if dedupe and n:
        _, first = np.unique(out, axis=0, return_index=True)
        out = out[np.sort(first)]
    return out


def gen_clusters(n: int, seed: int, k: int = 8, sigma: float = 0.02) -> np.ndarray:
    out = np.zeros((n, 3), dtype=np.float64)
    if n:
        library().d3g_gen_clusters(n, seed, k, sigma, _ptr(out))
    return out


def gen_lattice(n: int) -> np.ndarray:
    out = np.zeros((n, 3), dtype=np.float64)
    if n:
        library().d3g_gen_lattice(n, _ptr(out))
    return out


DISTRIBUTIONS = ("uniform", "clusters", "lattice", "sphere")


def gen_set(dist: str, n: int, seed: int) -> np.ndarray:
    """One set of the mixed workloads: n points of `dist` from `seed`."""
    if dist == "uniform":
        return gen_uniform(n, seed)
    if dist == "clusters":
        return gen_clusters(n, seed, 8, 0.02)
    if dist == "lattice":
        return gen_lattice(n)
    return gen_sphere(n, seed, 1.0, 1024, dedupe=True)


def partition_sets(sizes, n_parts: int, weights=None) -> List[List[int]]:
    """Splits independent point sets among `n_parts` GPUs (or streams) so that
    their build costs balance: longest-first greedy on the estimated cost
    n log2 n (times `weights[k]` if given - e.g. about 5 for integer lattices,
    whose degenerate cospherical cells cost more), each set to the least loaded
    part, ties to the lower part.  Deterministic; returns each part's set
    indices in ascending order.  Sets are independent, so the parts need no
    exchange step."""
    import heapq

    n_parts = int(n_parts)
    if n_parts < 1:
        raise ValueError("n_parts must be at least 1")
    sizes = np.asarray(sizes, dtype=np.float64).reshape(-1)
    w = np.ones_like(sizes) if weights is None else np.asarray(weights, dtype=np.float64).reshape(-1)
    if w.shape != sizes.shape:
        raise ValueError("weights must match sizes")
    cost = sizes * np.log2(np.maximum(sizes, 2.0)) * w
    order = np.argsort(-cost, kind="stable")
    heap = [(0.0, p) for p in range(n_parts)]
    parts: List[List[int]] = [[] for _ in range(n_parts)]
    for k in order.tolist():
        load, p = heapq.heappop(heap)
        parts[p].append(k)
        heapq.heappush(heap, (load + float(cost[k]), p))
    return [sorted(part) for part in parts]


def mixed_workload(n_sets: int, lo: int = 32, hi: int = 65536, seed: int = 2024, first_seed: int = 1000):
    """The mixed batched workload: n_sets sets with sizes log-uniform in
    [lo, hi] and a distribution drawn uniformly from DISTRIBUTIONS (both from
    numpy's PCG64 with `seed`); set k's points come from mt19937(first_seed + k)."""
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), n_sets))).astype(np.int64)
    dists = rng.integers(0, len(DISTRIBUTIONS), n_sets)
    return [gen_set(DISTRIBUTIONS[d], int(n), first_seed + k) for k, (n, d) in enumerate(zip(sizes, dists))]


# ---- input readers (host) -------------------------------------------------------------


def _mesh_arrays(m: "_Mesh"):
    v = np.ctypeslib.as_array(m.vertices, shape=(int(m.n_vertices) * 3,)).reshape(-1, 3).copy() \
        if m.n_vertices else np.zeros((0, 3), dtype=np.float64)
    f = np.ctypeslib.as_array(m.faces, shape=(int(m.n_faces) * 3,)).reshape(-1, 3).copy() \
        if m.n_faces else np.zeros((0, 3), dtype=np.int32)
    return v, f


def _path_bytes(path) -> bytes:
    return os.fsencode(path)


def load_mesh(path):
    """The reference viewer's reader (meshio::load, viewer/mesh_io.h:26-38): the
    format by extension - .obj, .off, .ply, .stl (welded), .xyz/.txt/.pts or
    none.  Returns (vertices (n, 3) float64, faces (m, 3) int32); raises
    Del3dError with the reference's error text when the reader fails."""
    lib = library()
    m = _Mesh()
    st = lib.d3g_mesh_load(_path_bytes(path), ctypes.byref(m))
    try:
        _check(st, "load_mesh")
        return _mesh_arrays(m)
    finally:
        lib.d3g_mesh_free(ctypes.byref(m))


def read_xyz(path) -> np.ndarray:
    """examples/simple.cpp:17-23: "x y z" triples until the first that does not
    parse; (n, 3) float64."""
    lib = library()
    m = _Mesh()
    st = lib.d3g_read_xyz(_path_bytes(path), ctypes.byref(m))
    try:
        _check(st, "read_xyz")
        return _mesh_arrays(m)[0]
    finally:
        lib.d3g_mesh_free(ctypes.byref(m))


def _mesh_in(vertices, faces):
    v = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 3).copy()
    f = np.ascontiguousarray(faces if faces is not None else np.zeros((0, 3)), dtype=np.int32).reshape(-1, 3).copy()
    m = _Mesh(v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), f.ctypes.data_as(ctypes.POINTER(_I32)),
              v.shape[0], f.shape[0])
    return v, f, m


def weld(vertices, faces=None):
    """meshio::weld: merges vertices with equal coordinates (first kept), remaps
    the faces and drops faces whose corners merged.  Returns (vertices, faces)."""
    v, f, m = _mesh_in(vertices, faces)
    _check(library().d3g_mesh_weld(ctypes.byref(m)), "weld")
    return v[:m.n_vertices].copy(), f[:m.n_faces].copy()


def drop_non_finite(vertices, faces=None):
    """meshio::drop_non_finite: removes vertices with a non-finite coordinate and
    the faces touching them.  Returns (vertices, faces, dropped)."""
    v, f, m = _mesh_in(vertices, faces)
    d = _I64(0)
    _check(library().d3g_mesh_drop_non_finite(ctypes.byref(m), ctypes.byref(d)), "drop_non_finite")
    return v[:m.n_vertices].copy(), f[:m.n_faces].copy(), d.value


def supported_formats() -> str:
    return library().d3g_mesh_supported_formats().decode()


def load_point_sets(paths, threads: int = 0):
    """Reads many files as point sets on host threads (faces ignored, non-finite
    vertices dropped) for a batched build.  Returns (xyz (N, 3) float64 with the
    sets back to back, set_offsets (n + 1,) int64, dropped (n,) int64); the sets
    are ``np.split(xyz, set_offsets[1:-1])``."""
    lib = library()
    enc = [_path_bytes(p) for p in paths]
    arr = (ctypes.c_char_p * max(len(enc), 1))(*enc)
    ps = _PointSets()
    _check(lib.d3g_load_point_sets(arr, len(enc), int(threads), ctypes.byref(ps)), "load_point_sets")
    try:
        n = int(ps.n_sets)
        offs = np.ctypeslib.as_array(ps.set_offsets, shape=(n + 1,)).copy()
        total = int(offs[-1])
        xyz = np.ctypeslib.as_array(ps.xyz, shape=(total * 3,)).reshape(-1, 3).copy() \
            if total else np.zeros((0, 3), dtype=np.float64)
        dropped = np.ctypeslib.as_array(ps.dropped, shape=(n,)).copy() if n else np.zeros(0, dtype=np.int64)
        return xyz, offs, dropped
    finally:
        lib.d3g_point_sets_free(ctypes.byref(ps))


# ---- checking a result (host) ---------------------------------------------------------


def validate_cells(all_cells, n_points: int = 0) -> None:
    """Checks all_cells() (infinite vertex -1) as the reference's Tds::validate()
    checks its cell table: distinct vertices in range, every facet shared by two
    consistently oriented cells, Euler characteristic 0 - necessary conditions,
    with no coordinates read (a complex flipped throughout, or not Delaunay,
    passes).  Raises Del3dError with the first violation.  Host only."""
    t = np.ascontiguousarray(all_cells, dtype=np.int32).reshape(-1, 4)
    _check(library().d3g_validate_cells(_ptr(t) if t.shape[0] else None, t.shape[0], int(n_points)),
           "validate_cells")
