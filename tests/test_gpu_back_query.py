"""GPU parity of FlashKNN.back_query (dense points -> nearest subset points).

Against the oracle: positions and FP32 distances bit-exact (ties by the lower
subset position).  Against the reference's own wrapper (golden fixtures from
tests/golden/make_golden_back.py) and, where the sm_100a build of the
reference kernels is present, against FlashKNN_Nearest_Back_Query_DL /
FlashKNN_Back_Query_DL on the GPU: the same neighbours with bit-identical
distances (the reference writes K > 1 rows in heap order and keeps the first
of equally near points).
"""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import ref_kernels
from tests.conftest import GOLDEN
from tests.test_oracle_golden import back_cases, same_up_to_kth_ties

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


def ours_vs_oracle(fk, xyz, sel, size, k, batch=None):
    gi, gd, empty = fk.ops.back_query(T(xyz), T(sel), size, k, None if batch is None else T(batch),
                                      validate=True)
    oi, od, oe = O.back_query(xyz, sel, size, k, batch)
    gi, gd = gi.cpu().numpy(), gd.cpu().numpy()
    assert np.array_equal(gi, oi)
    assert np.array_equal(gd.view(np.uint32), od.view(np.uint32))
    assert bool(empty) == bool(oe.any())
    return gi, gd


def sort_rows(idx, dist):
    """Rows ascending by distance (equal distances in any order)."""
    order = np.argsort(dist, 1, kind="stable")
    return np.take_along_axis(idx, order, 1), np.take_along_axis(dist, order, 1)


@pytest.mark.parametrize("case", back_cases())
def test_back_query_matches_reference_wrapper_and_oracle(fk, case):
    z = np.load(os.path.join(GOLDEN, f"back_{case}.npz"))
    k = int(z["k"])
    batch = z["batch"] if len(z["batch"]) else None
    gi, gd = ours_vs_oracle(fk, z["xyz"], z["sel"], float(z["query_grid_size"]), k, batch)
    if k == 1:
        assert np.array_equal(gi[:, 0], z["ref_idx"])
    else:
        ri, rd = sort_rows(z["ref_idx"], z["ref_dist"])
        assert same_up_to_kth_ties(gi, gd, ri, rd)


def test_back_query_wrapper_conventions(fk):
    z = np.load(os.path.join(GOLDEN, "back_uniform_k1.npz"))
    xyz, sel, size = T(z["xyz"]), T(z["sel"]), float(z["query_grid_size"])
    b = torch.zeros(len(z["xyz"]), dtype=torch.int64, device=DEV)
    one = fk.FlashKNN(num_nbr=1)
    out = one.back_query(xyz, sel, size, 0.08, b)
    assert out.dtype == torch.int64 and out.shape == (len(z["xyz"]),)
    assert np.array_equal(out.cpu().numpy(), z["ref_idx"])
    gm = one.back_query(xyz, sel, size, 0.08, b, memory_mode="GM")
    assert gm.shape == (len(z["xyz"]), 1) and torch.equal(gm[:, 0], out)
    idx, dist = fk.FlashKNN(num_nbr=8).back_query(xyz, sel, size, 0.08, b)
    assert idx.dtype == torch.int64 and idx.shape == (len(z["xyz"]), 8)
    assert torch.all(dist[:, 1:] >= dist[:, :-1])
    with pytest.raises(AssertionError):          # a cell with no subset point around it
        one.back_query(xyz, sel[:5], 0.01, 0.005, b)


@pytest.mark.parametrize("k", [1, 2, 4, 8, 16, 32])
def test_back_query_against_reference_kernels(fk, k):
    if not ref_kernels.available():
        pytest.skip("reference kernels not built (oracle/build_ref.py)")
    from oracle import ref_pipeline
    from flashknn_exprepo_b200 import synthetic as S
    xyz = S.room(target=30000)
    rng = np.random.default_rng(3)
    sel = np.sort(rng.choice(len(xyz), len(xyz) // 4, replace=False)).astype(np.int64)
    batch = np.zeros(len(xyz), np.int64)
    size = 0.2
    gi, gd = ours_vs_oracle(fk, xyz, sel, size, k, batch)
    ri, rd = ref_pipeline.reference_back_query(ref_kernels.load(), T(xyz), T(sel), size,
                                               T(batch), k)
    ri, rd = sort_rows(ri.cpu().numpy(), rd.cpu().numpy())
    assert same_up_to_kth_ties(gi, gd, ri, rd)


def test_back_query_large_batched(fk):
    from flashknn_exprepo_b200 import synthetic as S
    b = S.first_clouds(S.uneven_batch(), 3)
    batch = np.repeat(np.arange(3), b.counts).astype(np.int64)
    # subset: first point of every 10 cm voxel per cloud
    g = np.concatenate([np.floor(b.xyz / np.float32(0.1)).astype(np.int64), batch[:, None]], 1)
    _, first = np.unique(g, axis=0, return_index=True)
    sel = np.sort(first).astype(np.int64)
    for k in (1, 16):
        ours_vs_oracle(fk, b.xyz, sel, 0.2, k, batch)
