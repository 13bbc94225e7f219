"""The device spatial sort vs the reference: its rand48 shuffle, the 17 orders
the reference's own tests pin (FNV-1a hashes), and larger inputs vs the oracle."""
import numpy as np
import pytest
import torch

import del3d_b200 as d3
import oracle

pytestmark = pytest.mark.gpu

# tests/test_spatial_sort.cpp:115-147 of the reference.
PINNED_RANDOM = [(0, 0x14650fb0739d0383), (1, 0x315446a086a23133), (2, 0x29034675a49f07c2),
                 (5, 0x744ddb73fb935d27), (8, 0x7ec129e73709cb53), (9, 0x580cd772e82efaab),
                 (63, 0x18cf12b455d4e1ac), (64, 0x4fde96ee0b2e8be3), (65, 0xafa28526c6130f43),
                 (200, 0x23d15ee1f09fef23), (1000, 0x8b7191bde7a7449b)]
PINNED_OTHER = {
    "lattice 12x12x6": (lambda: oracle.ps_lattice(12, 12, 6), 0xdb779fbe6eb82833),
    "box shell 8": (lambda: oracle.ps_box_shell(8), 0x1667fe1e40586b6a),
    "300 identical": (lambda: np.tile([1.0, 2.0, 3.0], (300, 1)), 0xc9325f52533ad94f),
    "cylinder": (lambda: oracle.ps_cylinder(2000), 0x0b3b773499c64173),
    "sphere": (lambda: oracle.ps_sphere(2000), 0x93fb3414e085d46b),
    "torus": (lambda: oracle.ps_torus(2000), 0x0e117e42cb5f457f),
}


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 9, 63, 64, 65, 200, 1000, 70000, 1000000])
def test_shuffle_matches_reference_engine(cuda, n):
    out = torch.empty(n, dtype=torch.int32, device=cuda)
    st = d3.library().d3g_shuffle_device(n, out.data_ptr(), None)
    assert st == 0
    assert (out.cpu().numpy() == oracle.orc_shuffle(n)).all()


@pytest.mark.parametrize("n,h", PINNED_RANDOM)
def test_pinned_random(cuda, n, h):
    pts = oracle.ps_random_cube(n, 7)
    assert oracle.fnv1a_order(d3.spatial_sort(pts)) == h


@pytest.mark.parametrize("name", sorted(PINNED_OTHER))
def test_pinned_degenerate(cuda, name):
    make, h = PINNED_OTHER[name]
    assert oracle.fnv1a_order(d3.spatial_sort(make())) == h


@pytest.mark.parametrize("case", ["uniform_2e5", "lattice_30", "grid_dups", "sphere_q", "clusters"])
def test_matches_oracle(cuda, case):
    rng = np.random.default_rng(4)
    pts = {"uniform_2e5": lambda: d3.gen_uniform(200000, 3),
           "lattice_30": lambda: oracle.ps_lattice(30, 30, 30),
           "grid_dups": lambda: rng.integers(0, 12, (60000, 3)).astype(np.float64),
           "sphere_q": lambda: d3.gen_sphere(100000, 5, q=64, dedupe=False),
           "clusters": lambda: d3.gen_clusters(100000, 7)}[case]()
    assert (d3.spatial_sort(pts) == oracle.orc_spatial_sort(pts)).all()


def test_matches_reference_1e6(cuda):
    pts = d3.gen_uniform(1000000, 3)
    assert (d3.spatial_sort(pts) == oracle.ref_spatial_sort(pts)).all()


def test_matches_reference_multiblock_4e6(cuda):
    # Large enough that the top-level quickselects run as whole-GPU passes.
    pts = d3.gen_uniform(4000000, 8)
    assert (d3.spatial_sort(pts) == oracle.ref_spatial_sort(pts)).all()


def test_matches_reference_lattice_duplicates_large(cuda):
    # Many equal coordinates (long runs of ties in every quickselect).
    pts = np.random.default_rng(9).integers(0, 40, (600000, 3)).astype(np.float64)
    assert (d3.spatial_sort(pts) == oracle.ref_spatial_sort(pts)).all()
