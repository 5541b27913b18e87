"""GPU parity at the configuration sizes, against the reference kernel itself.

The reference's per-cloud pipeline -- its construction restated call by call
with the same ATen operations (oracle/ref_pipeline.py, after
FlashKNN/functions/FlashKnnWrapper.py:220-430) and its production kernel
FlashKNN_Query_Dynamic_Load (FlashKNN/csrc/flash_knn_query_dynamic_load.cu
:469-652) compiled for sm_100a by oracle/build_ref.py -- runs on the uniform
cube (16,384 points, K=16), the room (~80k points, K=32), the LiDAR scan
(~118k points, K=16, parent cells of 4 and 8 voxels) and on each of the 16
clouds of the uneven batch (1,464,355 points) at K=16 and K=32.  Our
FlashKNN.query runs on the same grid coordinates.

Criterion (the reference's own, Query/benchmark_thread_grouping.py:305-312):
bitwise-identical distance rows, and identical indices at every distance
below the row's K-th; at the K-th distance a tie may be resolved either way
(ours takes the lower index, the reference's network order decides its
choice).  The number of rows resolved differently is printed per case.

Also here: the batched query over the whole uneven batch equals the 16
plain per-cloud calls bit for bit (indices shifted by the cloud starts), at
K=16 and K=32.
"""
import numpy as np
import pytest
import torch

from flashknn_exprepo_b200 import synthetic as S
from oracle import ref_kernels

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_kernels.available(), reason="oracle/_ref not built")]

DEV = "cuda"


@pytest.fixture(scope="module")
def fk():
    import flashknn_exprepo_b200 as fk
    from flashknn_exprepo_b200.build import build
    build()
    return fk


@pytest.fixture(scope="module")
def batch():
    return S.uneven_batch()


def grid_of(xyz, voxel):
    # the FP32 product with the rounded reciprocal, as the offset entry points voxelise
    return np.floor(xyz * (np.float32(1) / np.float32(voxel))).astype(np.int64)


def compare_up_to_kth_ties(ours_i, ours_d, ref_i, ref_d):
    """Asserts the criterion above; returns the number of rows whose indices
    differ (only at ties at the K-th distance)."""
    assert ours_d.shape == ref_d.shape
    assert np.array_equal(ours_d.view(np.uint32), ref_d.view(np.uint32))
    rows = np.nonzero((ours_i != ref_i).any(1))[0]
    if len(rows) == 0:
        return 0
    d = ours_d[rows]
    a, b = ours_i[rows], ref_i[rows]
    sa = np.take_along_axis(a, np.lexsort((a, d), axis=-1), -1)
    sb = np.take_along_axis(b, np.lexsort((b, d), axis=-1), -1)
    below = d < d[:, -1:]  # rows are ascending: the sorted order keeps d in place
    bad = (sa != sb) & below
    assert not bad.any(), f"{int(bad.any(1).sum())} rows differ below the K-th distance"
    return len(rows)


def run_case(fk, xyz, voxel, num_down, k):
    from oracle import ref_pipeline
    cufun = ref_kernels.load()
    grid = torch.from_numpy(grid_of(xyz, voxel)).to(DEV)
    x = torch.from_numpy(np.ascontiguousarray(xyz)).to(DEV)
    zeros = torch.zeros(len(xyz), dtype=torch.int64, device=DEV)
    ri, rd = ref_pipeline.reference_query(cufun, grid, zeros, x, k, num_down)
    f = fk.FlashKNN(num_nbr=k, num_down=num_down)
    gi, gd = f.query(grid, None, x, return_distances=True, validate=True)
    return (gi.cpu().numpy().astype(np.int64), gd.cpu().numpy(), ri.cpu().numpy(),
            rd.cpu().numpy())


@pytest.mark.parametrize("name,k,num_down", [("cube", 16, 2), ("room", 32, 2),
                                             ("lidar", 16, 2), ("lidar", 16, 3)])
def test_single_cloud_configs_match_reference_kernel(fk, name, k, num_down):
    xyz, voxel = {"cube": (S.uniform_cube, S.C1_VOXEL), "room": (S.room, S.C2_VOXEL),
                  "lidar": (S.lidar, S.C3_VOXEL)}[name]
    xyz = xyz()
    gi, gd, ri, rd = run_case(fk, xyz, voxel, num_down, k)
    ties = compare_up_to_kth_ties(gi, gd, ri, rd)
    print(f"reference parity {name} K={k} alpha={1 << num_down}: {len(xyz)} rows, "
          f"{ties} resolved differently at a K-th-distance tie")


@pytest.mark.parametrize("k", [16, 32])
def test_every_uneven_batch_cloud_matches_reference_kernel(fk, batch, k):
    starts = np.concatenate([[0], batch.offsets[:-1]])
    total_ties = 0
    for c, (s, e) in enumerate(zip(starts, batch.offsets)):
        gi, gd, ri, rd = run_case(fk, batch.xyz[s:e], S.C4_VOXEL, 2, k)
        ties = compare_up_to_kth_ties(gi, gd, ri, rd)
        total_ties += ties
        print(f"reference parity uneven batch cloud {c} K={k}: {e - s} rows, {ties} ties")
    print(f"reference parity uneven batch K={k}: {len(batch.xyz)} rows, {total_ties} rows "
          f"resolved differently at a K-th-distance tie")


@pytest.mark.parametrize("k", [16, 32])
def test_batched_query_equals_per_cloud_calls(fk, batch, k):
    """One batched launch over the 16 clouds against the loop of 16 plain
    per-cloud calls (the comparator of the batched-vs-per-cloud speed-up)."""
    x = torch.from_numpy(batch.xyz).to(DEV)
    off = torch.from_numpy(batch.offsets).to(DEV)
    bi, bd = fk.ops.knn_offsets(x, off, k, S.C4_VOXEL, 2, validate=True)
    starts = np.concatenate([[0], batch.offsets[:-1]])
    for s, e in zip(starts.tolist(), batch.offsets.tolist()):
        ci, cd = fk.ops.knn_offsets(x[s:e].contiguous(),
                                    torch.tensor([e - s], dtype=torch.int64, device=DEV), k,
                                    S.C4_VOXEL, 2, validate=True)
        assert torch.equal(bi[s:e], ci + s), (s, e)
        assert torch.equal(bd[s:e].view(torch.int32), cd.view(torch.int32)), (s, e)


@pytest.mark.parametrize("name,k", [("room", 32), ("largest_cloud", 16)])
def test_table_abi_on_reference_built_tables(fk, batch, name, k):
    """The kernel-to-kernel comparison: the reference's tables (built by its
    own ATen construction) are equal to fknn_build_tables' bit for bit, and
    fknn_query_tables on them answers as FlashKNN_Query_Dynamic_Load does."""
    from oracle import ref_pipeline
    cufun = ref_kernels.load()
    if name == "room":
        xyz, voxel = S.room(), S.C2_VOXEL
    else:
        c = int(np.argmax(batch.counts))
        s = int(batch.offsets[c] - batch.counts[c])
        xyz, voxel = batch.xyz[s:int(batch.offsets[c])], S.C4_VOXEL
    grid = torch.from_numpy(grid_of(xyz, voxel)).to(DEV)
    x = torch.from_numpy(np.ascontiguousarray(xyz)).to(DEV)
    zeros = torch.zeros(len(xyz), dtype=torch.int64, device=DEV)
    t = ref_pipeline.reference_tables(cufun, grid, zeros, x, 2)
    ours = fk.ops.build_tables(grid, None, 2)
    # the same key sequence (the reference's argsort is unstable, so points
    # sharing a voxel may come in another order; with unique keys the orders
    # are equal)
    assert torch.equal(grid[ours["order"]], grid[t["order"]])
    for key in ("steps", "neigh", "cnt"):
        assert torch.equal(ours[key], t[key]), key
    n = len(xyz)
    ri = torch.zeros((n, k), dtype=torch.int32, device=DEV)
    rd = torch.zeros((n, k), dtype=torch.float32, device=DEV)
    cufun.FlashKNN_Query_Dynamic_Load(t["xyz_sorted"], t["steps"], t["neigh"], t["cnt"], k, ri,
                                      rd, 1, float("inf"))
    gi, gd = fk.ops.query_tables(t["xyz_sorted"], t["steps"], t["neigh"], t["cnt"], k,
                                 validate=True)
    ties = compare_up_to_kth_ties(gi.cpu().numpy(), gd.cpu().numpy(), ri.cpu().numpy(),
                                  rd.cpu().numpy())
    print(f"table ABI vs reference kernel, {name} K={k}: {n} rows, {ties} K-th-distance ties")
