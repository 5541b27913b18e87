"""GPU parity of the adaptive-neighbourhood query (AdaptiveNeighborhoodFlashKNN).

Against the oracle (same tie rule: lower input index): levels, indices and
FP32 distances bit-exact.  Against the reference's own pipeline (golden
fixtures from tests/golden/make_golden_adaptive.py): the same level for
every point, bit-identical distances, the same neighbours up to the order of
equal distances at the K-th place.
"""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.conftest import GOLDEN
from tests.test_oracle_golden import adaptive_args, adaptive_cases, same_up_to_kth_ties

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


def run(fk, grid, batch, k, xyz=None, min_factor=2, max_factor=8, max_shift=-1, cut_r2=np.inf):
    idx, dist, lv = fk.ops.adaptive_query(
        T(grid), None if batch is None else T(batch), k, xyz=None if xyz is None else T(xyz),
        min_factor=min_factor, max_factor=max_factor,
        max_shift=None if max_shift < 0 else max_shift, cut_r2=float(cut_r2), want_levels=True,
        validate=True)
    return idx.cpu().numpy(), dist.cpu().numpy(), lv.cpu().numpy().astype(np.int32)


def check_vs_oracle(fk, grid, batch, k, xyz=None, **kw):
    gi, gd, gl = run(fk, grid, batch, k, xyz, **kw)
    b = np.zeros(len(grid), np.int64) if batch is None else batch
    ol, oi, od = O.adaptive_query(grid, b, k, xyz, **kw)
    assert np.array_equal(gl, ol)
    assert np.array_equal(gi, oi)
    assert np.array_equal(gd.view(np.uint32), od.view(np.uint32))
    return gi, gd, gl


@pytest.mark.parametrize("case", adaptive_cases())
def test_adaptive_matches_reference_pipeline_and_oracle(fk, case):
    z = np.load(os.path.join(GOLDEN, f"adaptive_{case}.npz"))
    a = adaptive_args(z)
    k = a.pop("k")
    xyz = a.pop("xyz")
    gi, gd, gl = check_vs_oracle(fk, z["grid"], z["batch"], k, xyz, **a)
    assert np.array_equal(gl, z["ref_levels"])
    assert same_up_to_kth_ties(gi, gd, z["ref_idx"], z["ref_dist"])


def test_adaptive_wrapper_api(fk):
    z = np.load(os.path.join(GOLDEN, "adaptive_lidar_k16.npz"))
    knn = fk.AdaptiveNeighborhoodFlashKNN(num_nbr=16)
    idx = knn.query(T(z["grid"]), T(z["batch"]), T(z["xyz"]))
    assert idx.dtype == torch.int64 and idx.shape == (len(z["xyz"]), 16)
    idx2, dist = knn.query(T(z["grid"]), T(z["batch"]), T(z["xyz"]), return_distances=True)
    assert torch.equal(idx, idx2)
    assert same_up_to_kth_ties(idx.cpu().numpy(), dist.cpu().numpy(), z["ref_idx"],
                               z["ref_dist"])
    stats = knn.last_stats
    assert sum(stats["selected_level_points"].values()) == len(z["xyz"])


def test_c3_lidar_adaptive_full_size(fk):
    from flashknn_exprepo_b200 import synthetic as S
    xyz = S.lidar()
    grid = np.floor(xyz / np.float32(S.C3_VOXEL)).astype(np.int64)
    _, _, lv = check_vs_oracle(fk, grid, None, 16, xyz)
    assert len(np.unique(lv)) >= 3  # near field fine, far field coarse


def test_interleaved_batches_and_explicit_shift(fk):
    rng = np.random.default_rng(21)
    a = rng.random((3000, 3), dtype=np.float32)
    b = rng.random((1500, 3), dtype=np.float32) * np.float32(8) - np.float32(4)
    xyz = np.concatenate([a, b])
    batch = np.concatenate([np.full(3000, 7), np.full(1500, 2)]).astype(np.int64)
    perm = rng.permutation(len(xyz))
    xyz, batch = xyz[perm], batch[perm]
    grid = np.floor(xyz / np.float32(0.02)).astype(np.int64)
    check_vs_oracle(fk, grid, batch, 8, xyz)
    check_vs_oracle(fk, grid, batch, 8, xyz, max_shift=3)
    check_vs_oracle(fk, grid, batch, 12, None, min_factor=1, max_factor=3)


def test_adaptive_every_k_and_cut(fk):
    rng = np.random.default_rng(22)
    xyz = rng.random((5000, 3), dtype=np.float32) * np.float32(3)
    grid = np.floor(xyz / np.float32(0.05)).astype(np.int64)
    for k in (1, 5, 16, 32, 33, 64):
        check_vs_oracle(fk, grid, None, k, xyz)
    check_vs_oracle(fk, grid, None, 16, xyz, cut_r2=np.float32(0.01))


def test_adaptive_errors(fk):
    knn = fk.AdaptiveNeighborhoodFlashKNN(num_nbr=4)
    g = torch.zeros((10, 3), dtype=torch.int64, device=DEV)
    b = torch.zeros(10, dtype=torch.int64, device=DEV)
    with pytest.raises(ValueError):
        knn.query(g.cpu(), b.cpu())
    with pytest.raises(ValueError):
        knn.query(g[:3], b[:3])                      # fewer points than K
    with pytest.raises(ValueError):
        knn.query(g, b + 40000)                      # batch outside [0, 32768)
    wide = g.clone()
    wide[0, 0] = 70000                               # span >= 2^16
    with pytest.raises(ValueError):
        knn.query(wide, b)
    with pytest.raises(ValueError):
        knn.query(g, b, max_shift=17)
    idx = knn.query(g, b)                            # one voxel: everything ties at 0
    assert idx.shape == (10, 4)



def test_sparse_points_distinct_at_most_levels(fk):
    """Points spread over almost the whole coordinate range: nearly every
    point is a node of its own up to high octree levels, so the node count
    of all levels approaches its bound (n per level) and the node table runs
    at its highest load."""
    rng = np.random.default_rng(31)
    grid = rng.integers(0, 60000, (3000, 3)).astype(np.int64)
    xyz = grid.astype(np.float32) * np.float32(0.01)
    check_vs_oracle(fk, grid, None, 8, xyz)
    batch = rng.integers(0, 3, len(grid)).astype(np.int64)
    check_vs_oracle(fk, grid, batch, 4, xyz, min_factor=1, max_factor=2)
