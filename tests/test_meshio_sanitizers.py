"""The input readers under AddressSanitizer and UndefinedBehaviorSanitizer:
csrc/meshio.cpp is compiled with a small driver (tests/cpp/meshio_sanitize_driver.cpp)
and reads malformed files of every format - byte-level mutations of the reader
cases - and a large "x y z" file that is parsed in pieces on several threads.
Any report, crash or hang fails the test.  Host code only; no GPU."""
import os
import subprocess
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import meshio_cases as mc  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path, flags):
    exe = str(tmp_path / "drv")
    cmd = ["g++", "-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer", *flags,
           "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "meshio_sanitize_driver.cpp"),
           os.path.join(ROOT, "del3d_b200", "csrc", "meshio.cpp"), "-o", exe, "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip("sanitizer build unavailable: " + r.stderr[-300:])
    return exe


def test_readers_clean_under_address_and_ub_sanitizers(tmp_path):
    exe = _build(tmp_path, ["-fsanitize=address,undefined", "-fno-sanitize-recover=undefined"])
    files = mc.write_cases(str(tmp_path / "cases"), mc.mutated_cases(600, seed=99))
    files += mc.write_cases(str(tmp_path / "hand"), mc.hand_cases())
    big = b"".join(mc.random_xyz(__import__("numpy").random.default_rng(4)) for _ in range(1500))
    big_path = str(tmp_path / "big.xyz")
    with open(big_path, "wb") as fh:
        while fh.tell() < (5 << 20):
            fh.write(big)
    for k in range(0, len(files), 100):
        r = subprocess.run([exe] + files[k:k + 100], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0 and r.stdout.startswith("ok"), r.stderr[-3000:]
    r = subprocess.run([exe, big_path, big_path], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stderr[-3000:]


def test_threaded_loading_clean_under_thread_sanitizer(tmp_path):
    """d3g_load_point_sets on worker threads, and a large text file cut into
    pieces parsed on more threads inside them."""
    import numpy as np

    exe = _build(tmp_path, ["-fsanitize=thread"])
    rng = np.random.default_rng(8)
    chunk = b"".join(mc.random_xyz(rng) for _ in range(1500))
    big = []
    for k in range(3):
        p = str(tmp_path / f"big{k}.xyz")
        with open(p, "wb") as fh:
            while fh.tell() < (5 << 20):
                fh.write(chunk)
        big.append(p)
    small = mc.write_cases(str(tmp_path / "hand"), {k: v for k, v in mc.hand_cases().items() if not v.startswith(b"solid")})
    env = dict(os.environ, TSAN_OPTIONS="halt_on_error=1")
    r = subprocess.run([exe] + big + small, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0 and r.stdout.startswith("ok") and "WARNING: ThreadSanitizer" not in r.stderr, \
        r.stderr[-3000:]
