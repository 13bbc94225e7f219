"""The device rand48 shuffle (first stage of spatial_sort) vs the oracle."""
import numpy as np
import pytest
import torch

import del3d_b200 as d3
import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 9, 63, 64, 65, 200, 1000, 70000, 1000000])
def test_shuffle_matches_reference_engine(cuda, n):
    out = torch.empty(n, dtype=torch.int32, device=cuda)
    st = d3.library().d3g_shuffle_device(n, out.data_ptr(), None)
    assert st == 0
    assert (out.cpu().numpy() == oracle.orc_shuffle(n)).all()


def test_spatial_sort_is_permutation(cuda):
    pts = d3.gen_uniform(100000, 3)
    o = d3.spatial_sort(pts)
    assert (np.sort(o) == np.arange(len(pts))).all()
