"""Input readers (row f.4 of the scope): del3d_b200's host readers against the
reference viewer's reader (viewer/mesh_io.cpp, compiled from its source into
oracle/_ref/libmeshio_ref.so) on the same bytes, plus committed golden outputs
of that reader (tests/golden/meshio/, made by tests/golden/make_meshio_golden.py)
for machines without the reference tree.

Tolerance: none.  Vertices are compared bit for bit (as uint64), faces and
error texts exactly, and a file the reference fails on must fail here with the
same text and the same partial mesh.  No GPU is needed."""
import ctypes
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import del3d_b200 as d3
import oracle

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import meshio_cases as mc  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "meshio")

needs_ref = pytest.mark.skipif(not oracle.ref_meshio_available(), reason="oracle/_ref/libmeshio_ref.so not built")


def ours_raw(path):
    """d3g_mesh_load through the C ABI: (vertices, faces, error text or "")."""
    lib = d3.library()
    m = d3._Mesh()
    st = lib.d3g_mesh_load(os.fsencode(path), ctypes.byref(m))
    try:
        v, f = d3._mesh_arrays(m)
        err = lib.d3g_last_error().decode(errors="surrogateescape") if st != 0 else ""
        if st not in (0, 2):
            raise AssertionError(f"unexpected status {st} for {path}")
        return v, f, err
    finally:
        lib.d3g_mesh_free(ctypes.byref(m))


def same(a, b):
    v1, f1, e1 = a
    v2, f2, e2 = b
    return (v1.shape == v2.shape and np.array_equal(v1.view(np.uint64), v2.view(np.uint64))
            and np.array_equal(f1, f2) and e1 == e2)


def _compare_all(tmp_path, cases):
    paths = mc.write_cases(str(tmp_path), cases)
    bad = []
    for p in paths:
        ours, ref = ours_raw(p), oracle.ref_mesh_load(p)
        if not same(ours, ref):
            bad.append((os.path.basename(p), ours[2], ref[2], ours[0].shape, ref[0].shape, ours[1].shape,
                        ref[1].shape))
    assert not bad, bad[:5]
    return paths


@needs_ref
def test_hand_cases_match_reference(tmp_path):
    paths = _compare_all(tmp_path, mc.hand_cases())
    # the cases do reach every outcome
    errs = {oracle.ref_mesh_load(p)[2] for p in paths}
    for text in ("no points in the file", "no vertices in the OBJ", "empty OFF", "not an OFF file",
                 "malformed OFF header", "OFF ended inside the vertex list", "not a PLY file",
                 "PLY ended early", "PLY vertex element has no x/y/z", "no vertices in the PLY",
                 "PLY ended inside an element", "no triangles in the STL", "no vertices in the STL",
                 "truncated STL header"):
        assert text in errs, text
    assert any(e.startswith("unsupported PLY format") for e in errs)
    assert any(e.startswith("unknown extension") for e in errs)


@needs_ref
def test_random_cases_match_reference(tmp_path):
    _compare_all(tmp_path, mc.random_cases(n_each=40, seed=7))


@needs_ref
def test_mutated_files_match_reference(tmp_path):
    """Malformed files: every reader path on broken input.  Skipped per file:
    those on which the reference throws (it would abort a program) and welded
    STLs with a NaN vertex (the reference's weld orders vertices with operator<,
    undefined for NaN; here a NaN vertex never merges)."""
    paths = mc.write_cases(str(tmp_path), mc.mutated_cases(1200, seed=21))
    compared, bad = 0, []
    for p in paths:
        vr, fr, er, rc = oracle.ref_mesh_load(p, with_status=True)
        ours = ours_raw(p)
        if rc == 2 or (p.endswith(".stl") and (np.isnan(vr).any() or np.isnan(ours[0]).any())):
            continue
        compared += 1
        if not same(ours, (vr, fr, er)):
            bad.append((os.path.basename(p), ours[2], er, ours[0].shape, vr.shape))
    assert not bad, bad[:5]
    assert compared > 1100


@needs_ref
def test_large_xyz_in_pieces_matches_reference(tmp_path):
    """A text file above the piece size is parsed by several threads, cut at
    line starts; the points must be those of one pass."""
    rng = np.random.default_rng(31)
    chunks = [mc.random_xyz(rng) for _ in range(6000)]
    data = b"".join(chunks)
    big = b""
    while len(big) < (9 << 20):
        big += data
    p = str(tmp_path / "big.xyz")
    with open(p, "wb") as fh:
        fh.write(big)
    ours, ref = ours_raw(p), oracle.ref_mesh_load(p)
    assert ours[0].shape[0] > 100_000
    assert same(ours, ref)
    xyz, offs, _ = d3.load_point_sets([p], threads=4)      # one file, split four ways
    assert np.array_equal(xyz.view(np.uint64), d3.drop_non_finite(ref[0], None)[0].view(np.uint64))


@needs_ref
def test_missing_file_matches_reference(tmp_path):
    p = str(tmp_path / "absent.obj")
    assert same(ours_raw(p), oracle.ref_mesh_load(p))


def _random_mesh(rng, nv, nf, dup=0.3, nonfinite=0.0):
    base = rng.integers(-3, 4, size=(max(nv // 3, 1), 3)).astype(np.float64)
    v = rng.normal(size=(nv, 3))
    take = rng.random(nv) < dup
    v[take] = base[rng.integers(0, base.shape[0], int(take.sum()))]
    flip = rng.random(nv) < 0.1
    v[flip] = -v[flip] * (v[flip] == 0) + v[flip] * (v[flip] != 0)    # some -0.0
    if nonfinite:
        bad = rng.random((nv, 3)) < nonfinite
        v[bad] = rng.choice([np.nan, np.inf, -np.inf], int(bad.sum()))
    f = rng.integers(0, max(nv, 1), size=(nf, 3)).astype(np.int32) if nv else np.zeros((0, 3), np.int32)
    return v, f


@needs_ref
@pytest.mark.parametrize("seed", range(6))
def test_weld_matches_reference(seed):
    rng = np.random.default_rng(seed)
    v, f = _random_mesh(rng, int(rng.integers(0, 400)), int(rng.integers(0, 300)))
    ours = d3.weld(v, f)
    ref = oracle.ref_weld(v, f)
    assert np.array_equal(ours[0].view(np.uint64), ref[0].view(np.uint64))
    assert np.array_equal(ours[1], ref[1])


def test_weld_keeps_first_and_merges_signed_zero():
    v = np.array([[0.0, 1, 2], [-0.0, 1, 2], [3, 4, 5], [0.0, 1, 2], [7, 7, 7]])
    f = np.array([[0, 1, 2], [0, 2, 3], [2, 3, 0], [1, 2, 4]], np.int32)
    wv, wf = d3.weld(v, f)
    assert wv.tolist() == [[0, 1, 2], [3, 4, 5], [7, 7, 7]] and not np.signbit(wv[0, 0])
    assert wf.tolist() == [[0, 1, 2]]          # faces whose corners merged are gone
    # nothing equal: unchanged, degenerate faces kept
    v2 = np.array([[0.0, 0, 0], [1, 1, 1]])
    f2 = np.array([[0, 0, 1]], np.int32)
    wv2, wf2 = d3.weld(v2, f2)
    assert np.array_equal(wv2, v2) and np.array_equal(wf2, f2)
    # a NaN vertex never merges (the reference's ordering is undefined there)
    v3 = np.array([[np.nan, 0, 0], [np.nan, 0, 0]])
    assert d3.weld(v3, None)[0].shape == (2, 3)


@needs_ref
@pytest.mark.parametrize("seed", range(6))
def test_drop_non_finite_matches_reference(seed):
    rng = np.random.default_rng(100 + seed)
    v, f = _random_mesh(rng, int(rng.integers(0, 400)), int(rng.integers(0, 300)), nonfinite=0.02 * seed)
    ours = d3.drop_non_finite(v, f)
    ref = oracle.ref_drop_non_finite(v, f)
    assert np.array_equal(ours[0].view(np.uint64), ref[0].view(np.uint64))
    assert np.array_equal(ours[1], ref[1]) and ours[2] == ref[2]


@needs_ref
def test_supported_formats_match_reference():
    assert d3.supported_formats() == oracle.ref_mesh_formats()


def test_golden_outputs(tmp_path):
    """The reference reader's outputs, committed: parity without the reference tree."""
    with open(os.path.join(GOLDEN, "expected.json")) as fh:
        expected = json.load(fh)
    assert len(expected) >= 20
    for name, want in expected.items():
        v, f, err = ours_raw(os.path.join(GOLDEN, name))
        assert err == want["error"], name
        assert v.view(np.uint64).reshape(-1).tolist() == [int(x, 16) for x in want["vertex_bits"]], name
        assert f.reshape(-1).tolist() == want["faces"], name


def test_load_point_sets(tmp_path):
    cases = {k: v for k, v in mc.hand_cases().items()
             if k in ("plain.xyz", "quad.obj", "cube.off", "ascii.ply", "binary.ply", "binary.stl", "crlf.txt")}
    paths = mc.write_cases(str(tmp_path), cases)
    for threads in (1, 3, 0):
        xyz, offs, dropped = d3.load_point_sets(paths, threads=threads)
        assert offs.shape == (len(paths) + 1,) and offs[0] == 0 and offs[-1] == xyz.shape[0]
        for k, p in enumerate(paths):
            v, _ = d3.load_mesh(p)
            keep, _, nd = d3.drop_non_finite(v, None)
            assert dropped[k] == nd
            assert np.array_equal(xyz[offs[k]:offs[k + 1]].view(np.uint64), keep.view(np.uint64))
    assert np.isfinite(xyz).all()
    assert dropped.sum() > 0                 # binary.ply carries NaN / inf coordinates
    bad = mc.write_cases(str(tmp_path), {"broken.off": b"OFF\nno counts\n"})[0]
    with pytest.raises(d3.Del3dError, match="broken.off: malformed OFF header"):
        d3.load_point_sets(paths + [bad])
    assert d3.load_point_sets([])[1].tolist() == [0]


def test_read_xyz_stream_semantics(tmp_path):
    """examples/simple.cpp:17-23 reads triples until the first that fails."""
    p = tmp_path / "s.xyz"
    p.write_bytes(b"1 2 3 4\n5 6 # 7 8 9\n")
    assert d3.read_xyz(str(p)).tolist() == [[1, 2, 3], [4, 5, 6]]
    p.write_bytes(b"# comment first\n1 2 3\n")
    assert d3.read_xyz(str(p)).shape == (0, 3)
    with pytest.raises(d3.Del3dError):
        d3.read_xyz(str(tmp_path / "absent.xyz"))


def test_errors_raise_with_reference_text(tmp_path):
    p = tmp_path / "x.ply"
    p.write_bytes(b"ply\nformat binary_big_endian 1.0\nend_header\n")
    with pytest.raises(d3.Del3dError, match="unsupported PLY format 'binary_big_endian'"):
        d3.load_mesh(str(p))


def test_cpp_dropin_header_builds_and_runs(tmp_path):
    """A program written against the reference viewer's meshio interface links
    libdel3d_b200.so instead of viewer/mesh_io.cpp."""
    d3.library()
    src = tmp_path / "viewer_like.cpp"
    src.write_text(
        '#include "del3d/mesh_io.h"\n#include <cstdio>\n'
        "int main(int argc, char** argv) {\n"
        "  std::string err; meshio::Mesh m = meshio::load(argv[1], err);\n"
        "  std::size_t d = meshio::drop_non_finite(m); meshio::weld(m);\n"
        '  std::printf("%zu %zu %zu %s|%s\\n", m.vertices.size(), m.faces.size(), d, err.c_str(),\n'
        "              meshio::supported_formats());\n  return m.empty() ? 1 : 0;\n}\n")
    exe = tmp_path / "viewer_like"
    lib_dir = os.path.join(ROOT, "del3d_b200")
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-L", lib_dir,
                        "-ldel3d_b200", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    mesh = mc.write_cases(str(tmp_path), {"cube.off": mc.hand_cases()["cube.off"]})[0]
    out = subprocess.run([str(exe), mesh], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and out.stdout.strip() == "8 12 0 |obj, off, ply, stl, xyz", out.stdout


def test_bench_readers_workload_line():
    """bench.py --workload readers (host only) prints one JSON line whose points
    are the input's and, where the reference reader is built, the reference's."""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--workload", "readers", "--sets", "64",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["unit"] == "points/s" and line["value"] > 0 and line["sets_equal_input"]
    if oracle.ref_meshio_available():
        assert line["equals_reference"] and line["cpu_baseline"]["kind"] == "reference"


def test_c_abi_argument_errors():
    lib = d3.library()
    m = d3._Mesh()
    assert lib.d3g_mesh_load(None, ctypes.byref(m)) == 1
    assert lib.d3g_read_xyz(b"x.xyz", None) == 1
    assert lib.d3g_mesh_weld(None) == 1
    bad = d3._Mesh(None, None, 3, 0)                       # vertices missing
    assert lib.d3g_mesh_weld(ctypes.byref(bad)) == 1
    assert lib.d3g_mesh_drop_non_finite(ctypes.byref(bad), None) == 1
    v = np.zeros((2, 3))
    f = np.array([[0, 1, 5]], np.int32)                   # face index out of range
    mm = d3._Mesh(v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), f.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                  2, 1)
    assert lib.d3g_mesh_weld(ctypes.byref(mm)) == 2
    assert lib.d3g_mesh_drop_non_finite(ctypes.byref(mm), None) == 2
    ps = d3._PointSets()
    assert lib.d3g_load_point_sets(None, 2, 1, ctypes.byref(ps)) == 1
    assert lib.d3g_load_point_sets(None, 0, 1, None) == 1
    lib.d3g_mesh_free(None)
    lib.d3g_point_sets_free(None)
