"""knn_query_host (host buffers in, host buffers out, copies overlapped with
the query run by run) returns exactly what one device-side call returns."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fk():
    import flashknn_exprepo_b200 as fk
    from flashknn_exprepo_b200.build import build
    build()
    return fk


@pytest.mark.parametrize("chunks", [1, 3, 4, 40])
def test_host_query_equals_device_query(fk, chunks):
    from flashknn_exprepo_b200 import synthetic as S
    b = S.first_clouds(S.uneven_batch(), 6)
    xyz = torch.from_numpy(b.xyz).pin_memory()
    off = torch.from_numpy(b.offsets)
    idx, dist = fk.knn_query_host(16, xyz, off, voxel_size=S.C4_VOXEL, chunks=chunks)
    torch.cuda.current_stream().synchronize()
    di, dd = fk.ops.knn_offsets(xyz.cuda(), off.cuda(), 16, S.C4_VOXEL, 2)
    assert torch.equal(idx, di.cpu())
    assert torch.equal(dist.view(torch.int32), dd.cpu().view(torch.int32))


def test_host_query_into_caller_buffers(fk):
    rng = np.random.default_rng(2)
    xyz = torch.from_numpy(rng.random((5000, 3), dtype=np.float32)).pin_memory()
    off = torch.tensor([1000, 2500, 5000])
    idx = torch.full((5000, 8), -7, dtype=torch.int32).pin_memory()
    dist = torch.empty((5000, 8), dtype=torch.float32).pin_memory()
    out = fk.knn_query_host(8, xyz, off, idx, dist, voxel_size=0.02, chunks=2)
    torch.cuda.current_stream().synchronize()
    assert out[0] is idx and out[1] is dist
    di, dd = fk.ops.knn_offsets(xyz.cuda(), off.cuda(), 8, 0.02, 2)
    assert torch.equal(idx, di.cpu()) and torch.equal(dist, dd.cpu())


@pytest.mark.parametrize("chunks", [2, 4, 8])
def test_host_query_with_empty_clouds(fk, chunks):
    """Empty clouds (repeated ends) anywhere in the offsets, including whole
    runs of them: every run is still answered and placed by its offsets."""
    rng = np.random.default_rng(5)
    xyz = torch.from_numpy(rng.random((4000, 3), dtype=np.float32)).pin_memory()
    off = torch.tensor([0, 1000, 1000, 1000, 2500, 2500, 4000, 4000])
    idx, dist = fk.knn_query_host(8, xyz, off, voxel_size=0.02, chunks=chunks)
    torch.cuda.current_stream().synchronize()
    di, dd = fk.ops.knn_offsets(xyz.cuda(), off.cuda(), 8, 0.02, 2)
    assert torch.equal(idx, di.cpu())
    assert torch.equal(dist.view(torch.int32), dd.cpu().view(torch.int32))


@pytest.mark.parametrize("case", ["uniform_k16", "dense_multibatch_k64", "duplicate_voxels_k32"])
def test_traverse_info_is_the_mean_candidate_count(fk, case):
    """FlashKNN.query(traverse_info=...) writes the mean over parent cells of
    the points in their 27 neighbour cells, as the reference computes it from
    its tables (cnt_in_neigh[:, -1].float().mean(), FlashKnnWrapper.py:351-352)."""
    import os

    from tests.conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, f"tables_{case}.npz"))
    want = np.float32(z["ref_cnt"][:, 27].astype(np.float64).mean())
    info = [None]
    f = fk.FlashKNN(num_nbr=int(z["k"]), num_down=int(z["num_down"]))
    f.query(torch.from_numpy(z["grid"]).cuda(), torch.from_numpy(z["batch"]).cuda(),
            torch.from_numpy(z["xyz"]).cuda(), traverse_info=info)
    assert info[0] == pytest.approx(float(want), rel=1e-6)


def test_graph_mode_replays_the_eager_pipeline(fk):
    """graph=True: the first call captures, later calls replay; the results
    equal the eager call's bit for bit, also after the input values change
    in place (same pointers, same graph) and for a second input."""
    from flashknn_exprepo_b200 import synthetic as S
    xyz = torch.from_numpy(S.uniform_cube()).cuda()
    off = torch.tensor([xyz.shape[0]], device="cuda")
    want = fk.ops.knn_offsets(xyz, off, 16, S.C1_VOXEL, 2)
    for _ in range(3):
        got = fk.ops.knn_offsets(xyz, off, 16, S.C1_VOXEL, 2, graph=True, validate=True)
        assert torch.equal(got[0], want[0]) and torch.equal(got[1], want[1])
    xyz.mul_(0.5).add_(0.25)  # new values at the same address: the same graph
    want = fk.ops.knn_offsets(xyz, off, 16, S.C1_VOXEL, 2)
    got = fk.ops.knn_offsets(xyz, off, 16, S.C1_VOXEL, 2, graph=True)
    assert torch.equal(got[0], want[0]) and torch.equal(got[1], want[1])
    grid = torch.floor(xyz / S.C1_VOXEL).long()
    f = fk.FlashKNN(num_nbr=8, num_down=2)
    want = f.query(grid, None, xyz)
    for _ in range(2):
        assert torch.equal(f.query(grid, None, xyz, graph=True), want)
