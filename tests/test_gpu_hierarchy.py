"""GPU parity of voxel-first subsampling and the DeLA hierarchy builder.

Against the oracle: identical index arrays.  Against the reference's own
Networks/hierarchy.py (golden fixtures from
tests/golden/make_golden_hierarchy.py): every output tensor identical.
"""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.conftest import GOLDEN
from tests.test_oracle_golden import hierarchy_cases

pytestmark = pytest.mark.gpu

DEV = "cuda"


@pytest.fixture(scope="module")
def fk():
    import flashknn_exprepo_b200 as fk
    from flashknn_exprepo_b200.build import build
    build()
    return fk


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


@pytest.mark.parametrize("case", hierarchy_cases())
def test_hierarchy_matches_reference_builder(fk, case):
    z = np.load(os.path.join(GOLDEN, f"hierarchy_{case}.npz"))
    sizes = tuple(float(s) for s in z["voxel_sizes"])
    ks = tuple(int(k) for k in z["ks"])
    xyz = T(z["xyz"])
    for i, s in enumerate(sizes):
        assert np.array_equal(fk.hierarchy.voxel_first(xyz, s).cpu().numpy(),
                              z[f"voxel_first_{i}"])
    outs = fk.hierarchy.build_flash_hierarchy(xyz, sizes, ks, int(z["alpha"]))
    assert len(outs) == int(z["n_outputs"])
    for i, o in enumerate(outs):
        assert o.dtype == torch.int64
        assert np.array_equal(o.cpu().numpy(), z[f"ref_{i}"]), i


def test_voxel_first_vs_oracle_full_size(fk):
    from flashknn_exprepo_b200 import synthetic as S
    b = S.uneven_batch()
    xyz = b.xyz
    for size in (0.05, 0.06, 0.12, 0.3):              # any size: reciprocal rounding
        got = fk.ops.voxel_first(T(xyz), size, validate=True).cpu().numpy()
        assert np.array_equal(got, O.voxel_first(xyz, size))
    batch = np.repeat(np.arange(len(b.counts)), b.counts).astype(np.int64)
    got = fk.ops.voxel_first(T(xyz), 0.2, T(batch), validate=True).cpu().numpy()
    assert np.array_equal(got, O.voxel_first(xyz, 0.2, batch))


def test_voxel_first_edges(fk):
    empty = fk.ops.voxel_first(torch.zeros((0, 3), device=DEV), 0.1)
    assert empty.numel() == 0
    pts = np.array([[0.0, 0, 0], [0.01, 0.01, 0.01], [-0.01, 0, 0], [5, 5, 5], [5, 5, 5]],
                   np.float32)
    got = fk.ops.voxel_first(T(pts), 0.1).cpu().numpy()
    assert got.tolist() == [0, 2, 3]                  # floor: -0.01 is its own voxel
    with pytest.raises(fk.FknnError):
        fk.ops.voxel_first(T(pts), 0.1, T(np.array([0, 0, 0, 0, 40000])), validate=True)


def test_hierarchy_default_sizes_on_a_lidar_scan(fk):
    from flashknn_exprepo_b200 import synthetic as S
    xyz = S.lidar(dedup=True)
    outs = fk.hierarchy.build_flash_hierarchy(T(xyz))
    assert len(outs) == 10
    # the oracle's composition of the same steps
    from tests.test_oracle_golden import oracle_hierarchy
    want = oracle_hierarchy(xyz, (0.06, 0.12, 0.24, 0.48), (24, 24, 24, 24), 16)
    for i, (o, w) in enumerate(zip(outs, want)):
        assert np.array_equal(o.cpu().numpy(), w), i
