"""The C ABI library loads and exports every entry point include/*.h declares
(no GPU needed; no compute calls)."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT

import del3d_b200


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b(?:int|void|const char\*)\s+(d3g_\w+)\s*\(", text):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "d3g_build" in names and "d3g_predicates" in names and "d3g_spatial_sort" in names


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(name):
    lib = del3d_b200.library()
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_status_strings():
    lib = del3d_b200.library()
    assert lib.d3g_status_string(0) == b"ok"
    assert lib.d3g_status_string(4) == b"exact-stage capacity exceeded"
    assert lib.d3g_predicate_arity(0) == 4 and lib.d3g_predicate_arity(1) == 5
    assert lib.d3g_predicate_arity(99) == 0


def test_bad_arguments_rejected_without_device():
    lib = del3d_b200.library()
    # Null output / negative sizes are rejected before any device work.
    assert lib.d3g_build(None, -1, None, None) == 1
    assert lib.d3g_predicates(None, 0, None, -5, 0, None, None) == 1


def test_memory_calls_without_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    # Releasing the caches and reading the pool need a device; both report it.
    with pytest.raises(del3d_b200.Del3dError):
        del3d_b200.release_cached_memory()
    with pytest.raises(del3d_b200.Del3dError):
        del3d_b200.pool_usage()
