"""GPU: fknn_query_tables_noalloc, the table query that allocates nothing.

Some callers cannot give the library device memory -- a plugin whose host
framework owns every device allocation, a real-time loop that must not
allocate after start-up, a binding that only forwards tensors.  For them the
entry point keeps its scratch in a fixed array inside the library.  This
file checks it through the C ABI against fknn_query_tables (which takes a
caller workspace) on consecutive calls, whose shared scratch still holds the
previous call's contents, and checks the size limit.  It is collected last
so that a failure here leaves every other test already run.
"""
import ctypes
import os

import numpy as np
import pytest
import torch

from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu

DEV = "cuda"


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def tables(case):
    z = np.load(os.path.join(GOLDEN, f"tables_{case}.npz"))
    return (T(z["ref_xyz_sorted"]), T(z["ref_steps"]), T(z["ref_neigh"]), T(z["ref_cnt"]),
            int(z["k"]))


def call_noalloc(lib, xyz, steps, neigh, cnt, k, cut_r2=float("inf")):
    n, p = xyz.shape[0], neigh.shape[0]
    idx = torch.full((n, k), -7, dtype=torch.int32, device=DEV)
    dist = torch.full((n, k), float("nan"), dtype=torch.float32, device=DEV)
    rc = lib.fknn_query_tables_noalloc(xyz.data_ptr(), n, steps.data_ptr(), neigh.data_ptr(),
                                       cnt.data_ptr(), p, k, cut_r2, idx.data_ptr(),
                                       dist.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return rc, idx, dist


def test_noalloc_matches_workspace_entry_point_on_consecutive_calls():
    from flashknn_exprepo_b200 import _lib, ops
    from flashknn_exprepo_b200.build import build
    build()
    lib = _lib.load()
    # a larger problem, then a smaller one twice: the scratch still holds the
    # previous call's data when the next one starts
    for case in ["dense_multibatch_k64", "uniform_k16", "uniform_k16", "duplicate_voxels_k32"]:
        xyz, steps, neigh, cnt, k = tables(case)
        want_idx, want_dist = ops.query_tables(xyz, steps, neigh, cnt, k)
        for _ in range(2):
            rc, idx, dist = call_noalloc(lib, xyz, steps, neigh, cnt, k)
            assert rc == _lib.FKNN_OK, lib.fknn_error_string(rc)
            torch.cuda.synchronize()
            assert torch.equal(idx, want_idx), case
            # same distances bit for bit (well within any FP32 tolerance)
            assert torch.equal(dist.view(torch.int32), want_dist.view(torch.int32)), case


def test_noalloc_rejects_problems_beyond_its_scratch():
    from flashknn_exprepo_b200 import _lib
    lib = _lib.load()
    xyz, steps, neigh, cnt, k = tables("uniform_k16")
    too_many = 32769
    rc = lib.fknn_query_tables_noalloc(xyz.data_ptr(), too_many, steps.data_ptr(),
                                       neigh.data_ptr(), cnt.data_ptr(), neigh.shape[0], k,
                                       float("inf"), None, None,
                                       torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.FKNN_ERR_SCRATCH_LIMIT
    assert b"scratch" in lib.fknn_error_string(rc)
