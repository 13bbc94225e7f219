"""The C++ drop-in: include/del3d/*.h (the reference's declarations) implemented
by libdel3d_b200.so.

* tests/cpp/dropin_check.cpp, a caller written against the reference's
  interface, compiles and links here (CPU) and, on the GPU, returns what the
  Python API and the reference return.
* The reference's own test programs (tests/test_*.cpp) and example, compiled
  against the drop-in by oracle/Makefile into oracle/_ref/dropin/, pass on the
  GPU - except test_delaunay's pinned cell-allocation-order hashes, the one
  documented difference (cells come back in canonical order).
"""
import os
import subprocess

import numpy as np
import pytest

import del3d_b200 as d3
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "dropin_check.cpp")
DROPIN = os.path.join(ROOT, "oracle", "_ref", "dropin")


def _compile(out_path):
    lib_dir = os.path.join(ROOT, "del3d_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), SRC, "-L", lib_dir,
           "-ldel3d_b200", f"-Wl,-rpath,{lib_dir}", "-o", out_path]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_dropin_compiles_and_links(tmp_path):
    d3.library()                      # the library is built
    _compile(str(tmp_path / "dropin_check"))


@pytest.mark.gpu
def test_dropin_matches_python_api_and_reference(cuda, tmp_path):
    exe = str(tmp_path / "dropin_check")
    _compile(exe)
    n, seed = 3000, 17
    r = subprocess.run([exe, str(n), str(seed), str(tmp_path)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr

    def load(name, dt, cols=None):
        a = np.fromfile(str(tmp_path / name), dtype=dt)
        return a.reshape(-1, cols) if cols else a

    pts = d3.gen_uniform(n, seed)
    d = d3.Delaunay()
    d.build(pts)
    cells = load("cells.i32", np.int32, 4)
    assert np.array_equal(cells, d.finite_cells())
    assert np.array_equal(load("all.i32", np.int32, 4), d.all_cells())
    assert np.array_equal(load("incident_sizes.i32", np.int32), np.diff(d.incident_csr()[0]))
    assert int(load("nvertices.i64", np.int64)[0]) == d.number_of_vertices()
    if oracle.ref_available():
        want = oracle.canonical_cells(oracle.ref_build(pts)["cells"])
        assert np.array_equal(cells, want)

    k = min(64, cells.shape[0])
    t = cells[:k]
    assert np.array_equal(load("cc.f64", np.float64, 3), d3.circumcenters(pts, t))
    assert np.array_equal(load("ccl.f64", np.float64, 3), d3.circumcenters(pts, t, lazy=True))
    signs = load("signs.i32", np.int32).reshape(k, 3)
    assert np.array_equal(signs[:, 0], d3.orient3d(pts, t))
    assert np.array_equal(signs[:, 1], d3.in_sphere(pts, np.c_[t, t[:, 0]]))
    e = (np.arange(k) * 7) % n
    assert np.array_equal(signs[:, 2], d3.in_sphere_unperturbed(pts, np.c_[t, e]))
    assert np.array_equal(load("order.i32", np.int32), d3.spatial_sort(pts))


def _run_reference_program(name, timeout=900):
    exe = os.path.join(DROPIN, name)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built (oracle/Makefile, needs the reference tree)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=timeout, cwd=DROPIN)
    return r.returncode, r.stdout + r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name,banner", [
    ("test_predicates", "ALL PREDICATES MATCH THE REFERENCE"),
    ("test_predicates2", "ALL COPLANAR PREDICATES MATCH THE REFERENCE"),
    ("test_spatial_sort", "THE ORDER IS THE PINNED ONE"),
])
def test_reference_test_programs_pass(cuda, name, banner):
    rc, out = _run_reference_program(name)
    assert rc == 0 and banner in out, out[-3000:]


@pytest.mark.gpu
def test_reference_delaunay_test_only_order_differs(cuda):
    rc, out = _run_reference_program("test_delaunay")
    fails = [ln.strip() for ln in out.splitlines() if ln.strip().startswith("FAIL:")]
    # Every property check holds (orientation, empty circumspheres, facet
    # closure, vertex counts, incident lists, determinism); what fails is the
    # pinned allocation-order hash of the 11 pinned cases (a tiny case whose
    # allocation order happens to be the canonical one may still match).
    assert all(f == "FAIL: cell sequence differs from the pinned value" for f in fails), fails
    assert 1 <= len(fails) <= 11, out[-3000:]
    assert rc == 1


@pytest.mark.gpu
def test_reference_example_runs(cuda):
    rc, out = _run_reference_program("simple")
    assert rc == 0, out[-3000:]
