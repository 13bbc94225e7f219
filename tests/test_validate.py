"""d3g_validate_cells, the output-side counterpart of the reference's
Tds::validate() (src/tds.h:483-530): the reference's own all_cells() outputs
must pass - in allocation order, reversed, and in the canonical form this
library returns - and every kind of corruption must fail.  Host only."""
import numpy as np
import pytest

import del3d_b200 as d3
import oracle

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


def _sets():
    return [("uniform", d3.gen_uniform(3000, 1)), ("lattice", d3.gen_lattice(1000).astype(np.float64)),
            ("clusters", d3.gen_clusters(2000, 2)), ("sphere", d3.gen_sphere(1500, 3, 1.0, 1024, dedupe=True)),
            ("tet", np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]])),
            ("duplicates", np.repeat(d3.gen_uniform(200, 9), 3, axis=0))]


def _invalid(cells, n_points=0, match=None):
    with pytest.raises(d3.Del3dError, match=match):
        d3.validate_cells(cells, n_points)


@needs_ref
@pytest.mark.parametrize("name,pts", _sets(), ids=[n for n, _ in _sets()])
def test_reference_outputs_are_valid(name, pts):
    cells = oracle.ref_build(pts)["all"]
    n = pts.shape[0]
    d3.validate_cells(cells, n)
    d3.validate_cells(cells[::-1], n)
    d3.validate_cells(oracle.canonical_cells(cells), n)        # the form this library returns


@needs_ref
def test_corruptions_are_caught():
    pts = d3.gen_uniform(500, 4)
    good = oracle.ref_build(pts)["all"]
    n = pts.shape[0]
    finite = np.flatnonzero((good >= 0).all(axis=1))
    k = int(finite[7])

    bad = good.copy()
    bad[k, [0, 1]] = bad[k, [1, 0]]                               # odd permutation: orientation flipped
    _invalid(bad, n, "not consistently oriented")
    bad = good.copy()
    bad[k] = bad[k, [1, 2, 0, 3]]                                 # even rotation: still valid
    d3.validate_cells(bad, n)
    _invalid(np.delete(good, k, axis=0), n, "belongs to 1 cells")  # a missing cell
    _invalid(np.vstack([good, good[k:k + 1]]), n, "belongs to")    # a cell twice
    bad = good.copy()
    bad[k, 1] = bad[k, 0]
    _invalid(bad, n, "repeats vertex")
    bad = good.copy()
    bad[k, 2] = n + 5
    _invalid(bad, n, "out of range")
    d3.validate_cells(good, 0)                                    # no upper bound given: range unchecked
    bad = good.copy()
    bad[k, 3] = -7
    _invalid(bad, 0, "out of range")
    inf = int(np.flatnonzero((good < 0).any(axis=1))[0])
    bad = good.copy()
    bad[inf] = np.where(bad[inf] >= 0, bad[inf], -1)
    j = int(np.flatnonzero(bad[inf] >= 0)[0])
    bad[inf, j] = -1
    _invalid(bad, n, "repeats vertex|more than one infinite")
    # two copies glued at the infinite vertex: every facet matched, but not a sphere
    twin = np.where(good >= 0, good + n, -1)
    _invalid(np.vstack([good, twin]), 2 * n, "Euler characteristic -1")


def test_empty_and_bad_arguments():
    d3.validate_cells(np.zeros((0, 4), np.int32))                 # no cells (degenerate input): nothing to check
    lib = d3.library()
    assert lib.d3g_validate_cells(None, 5, 0) == 1
    assert lib.d3g_validate_cells(None, -1, 0) == 1
