"""GPU parity of neighbour grouping (grouping / knn_query_and_group).

Forward: the gathered rows equal Pointcept's own grouping output exactly
(it is a copy plus one FP32 subtraction).  Backward: the hand-written
deterministic gradients equal torch autograd's (Pointcept fixtures) and an
FP64 restatement within 1e-5 relative, and are bitwise identical run to run.
"""
import os

import numpy as np
import pytest
import torch

from tests.conftest import GOLDEN
from tests.test_oracle_golden import grouping_cases, grouping_f64

pytestmark = pytest.mark.gpu

DEV = "cuda"


@pytest.fixture(scope="module")
def fk():
    import flashknn_exprepo_b200 as fk
    from flashknn_exprepo_b200.build import build
    build()
    return fk


def T(a, grad=False):
    t = torch.from_numpy(np.ascontiguousarray(a)).to(DEV)
    return t.requires_grad_(True) if grad else t


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


def run_case(fk, z):
    with_xyz, separate = bool(z["with_xyz"]), bool(z["separate"])
    feat, xyz = T(z["feat"], True), T(z["xyz"], with_xyz)
    new = T(z["new_xyz"], True) if separate else None
    out = fk.grouping(T(z["idx"]), feat, xyz, new, with_xyz=with_xyz)
    (out * T(z["grad_out"])).sum().backward()
    grads = {"feat": feat.grad.cpu().numpy()}
    if with_xyz:
        grads["xyz"] = xyz.grad.cpu().numpy()
        if separate:
            grads["new_xyz"] = new.grad.cpu().numpy()
    return out.detach().cpu().numpy(), grads


@pytest.mark.parametrize("case", grouping_cases())
def test_grouping_matches_pointcept(fk, case):
    z = np.load(os.path.join(GOLDEN, f"grouping_{case}.npz"))
    out, grads = run_case(fk, z)
    assert np.array_equal(out, z["ref_out"])
    _, want = grouping_f64(z)
    assert rel(grads["feat"], z["ref_grad_feat"]) <= 1e-5
    assert rel(grads["feat"], want["feat"]) <= 1e-5
    for key in ("xyz", "new_xyz"):
        if key in grads:
            assert rel(grads[key], want[key]) <= 1e-5
            assert rel(grads[key], z[f"ref_grad_{key}"]) <= 1e-5
    out2, grads2 = run_case(fk, z)                   # bitwise reproducible
    for key in grads:
        assert np.array_equal(grads[key].view(np.uint32), grads2[key].view(np.uint32))


def test_hub_points_long_segments(fk):
    rng = np.random.default_rng(9)
    n, m, k, c = 500, 400, 16, 20
    idx = rng.integers(0, n, (m, k)).astype(np.int32)
    idx[:, 0] = 7                                    # point 7: 400 entries
    idx[::2, 1] = 11                                 # point 11: 200 entries
    z = {"idx": idx, "feat": rng.standard_normal((n, c)).astype(np.float32),
         "xyz": rng.random((n, 3), dtype=np.float32),
         "new_xyz": rng.random((m, 3), dtype=np.float32),
         "grad_out": rng.standard_normal((m, k, c + 3)).astype(np.float32),
         "with_xyz": np.bool_(True), "separate": np.bool_(True)}
    out, grads = run_case(fk, z)
    ref_out, want = grouping_f64(z)
    assert np.array_equal(out, ref_out.astype(np.float32))
    for key in ("feat", "xyz", "new_xyz"):
        assert rel(grads[key], want[key]) <= 1e-5


def test_knn_query_and_group_full_size(fk):
    from flashknn_exprepo_b200 import synthetic as S
    b = S.first_clouds(S.uneven_batch(), 6)
    xyz, offs = T(b.xyz), T(b.offsets)
    feat = torch.randn((len(b.xyz), 64), device=DEV)
    grouped, idx = fk.knn_query_and_group(feat, xyz, offs, nsample=16, with_xyz=True,
                                          voxel_size=S.C4_VOXEL)
    il = idx.long()
    want = torch.cat([xyz[il] - xyz[:, None, :], feat[il]], -1)
    assert torch.equal(grouped, want)
    plain, idx2 = fk.knn_query_and_group(feat, xyz, offs, idx=idx, with_xyz=False)
    assert torch.equal(plain, feat[il]) and idx2 is idx
