"""GPU parity of the radius-limited grid query (fknn_ball_query / ball_query).

Against the oracle (the grid kNN with cut radius, padding -1): indices and
FP32 squared distances bit-exact.  With the default voxel (parent cell =
radius) the rows equal an exact within-radius top-K over the whole cloud,
checked against the oracle run with one cell holding every point.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O

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


def oracle_ball(xyz, offs, k, r, voxel, num_down=2, q=None, qoffs=None):
    r2 = np.float32(r) * np.float32(r)
    oi, od = O.knn_offsets(xyz, offs, k, voxel, num_down, new_xyz=q, new_offsets=qoffs, cut_r2=r2)
    return np.where(np.isinf(od), -1, oi), od


def test_ball_query_room_self_vs_oracle_and_exact(fk):
    from flashknn_exprepo_b200 import synthetic as S
    xyz = S.room(target=40000)
    offs = np.array([len(xyz)])
    padded = full = False
    for k, r in ((32, 0.1), (16, 0.05), (8, 0.3)):
        gi, gd = fk.ops.ball_query_offsets(T(xyz), T(offs), k, r, r / 4, 2, validate=True)
        gi, gd = gi.cpu().numpy(), gd.cpu().numpy()
        oi, od = oracle_ball(xyz, offs, k, r, r / 4)
        assert np.array_equal(gi, oi)
        assert np.array_equal(gd.view(np.uint32), od.view(np.uint32))
        # exact: one cell holding every point gives the within-radius top-K
        ei, ed = oracle_ball(xyz, offs, k, r, 1e4)
        assert np.array_equal(gi, ei)
        assert np.all(gd[gi >= 0] < np.float32(r) * np.float32(r))
        padded |= bool((gi < 0).any())
        full |= bool((gi >= 0).all(1).any())
    assert padded and full  # both small balls (padding) and full rows occur


def test_ball_query_pointcept_convention_multi_cloud_general(fk):
    from flashknn_exprepo_b200 import synthetic as S
    b = S.first_clouds(S.uneven_batch(), 4)
    xyz, offs = b.xyz, b.offsets
    rng = np.random.default_rng(5)
    qcloud = np.sort(rng.integers(0, 4, 5000))
    # queries near the points of their own cloud, in cloud order
    starts = np.concatenate([[0], offs[:-1]])
    q = np.concatenate([xyz[rng.integers(s, e, (qcloud == c).sum())]
                        + rng.normal(0, 0.05, ((qcloud == c).sum(), 3)).astype(np.float32)
                        for c, (s, e) in enumerate(zip(starts, offs))]).astype(np.float32)
    qoffs = np.cumsum(np.bincount(qcloud, minlength=4))
    idx, dist = fk.ball_query(24, 0.2, 0.0, T(xyz), T(offs), T(q), T(qoffs))
    assert idx.dtype == torch.int32 and idx.shape == (len(q), 24)
    idx, dist = idx.cpu().numpy(), dist.cpu().numpy()
    oi, od = oracle_ball(xyz, offs, 24, 0.2, 0.2 / 4, q=q, qoffs=qoffs)
    assert np.array_equal(idx, oi)
    assert np.array_equal(dist[idx >= 0], np.sqrt(od[oi >= 0]))
    assert np.all(dist[idx < 0] == np.float32(1e5))   # sqrt of the 1e10 padding
    self_idx, _ = fk.ball_query(8, 0.1, 0.0, T(xyz), T(offs))
    assert (self_idx[:, 0].cpu().numpy() >= 0).all()
    with pytest.raises(ValueError):
        fk.ball_query(8, 0.1, 0.05, T(xyz), T(offs))
