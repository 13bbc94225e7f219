"""d3g_autotune_device: picks the fastest speed setting on a sample and makes it
the device's default; the cells do not depend on the setting."""
import numpy as np
import pytest

import del3d_b200 as d3

pytestmark = pytest.mark.gpu


def test_autotune_picks_a_setting_and_cells_do_not_change(cuda):
    import torch

    sets = d3.mixed_workload(48, lo=32, hi=8192, seed=5, first_seed=300)
    offs = np.zeros(len(sets) + 1, dtype=np.int64)
    offs[1:] = np.cumsum([a.shape[0] for a in sets])
    x = torch.from_numpy(np.concatenate(sets)).to(cuda)
    d3.reset_tuning()
    before, co0, nv0 = d3.build_batch_device(x, offs)
    before = before.clone()
    try:
        t = d3.autotune(x, offs)
        assert t["candidates"] == 10 and t["ms"] > 0
        assert t["schedule"] in (0, 1) and t["chunk"] < 0 and t["alpha_small"] > 0
        assert d3.get_tuning()["chunk"] == t["chunk"]
        after, co1, nv1 = d3.build_batch_device(x, offs)      # tuned defaults
        assert torch.equal(after, before) and np.array_equal(co0, co1) and np.array_equal(nv0, nv1)
    finally:
        d3.reset_tuning()
    assert d3.get_tuning()["candidates"] == 0
