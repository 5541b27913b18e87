"""GPU: fknn_query_tables_noalloc, the table query that allocates nothing.

Some callers cannot give the library device memory -- a plugin whose host
framework owns every device allocation, a real-time loop that must not
allocate after start-up, a binding that only forwards tensors.  For them the
entry point keeps its scratch in a fixed array inside the library.  This
file checks it through the C ABI against fknn_query_tables (which takes a
caller workspace) on consecutive calls, whose shared scratch still holds the
previous call's contents, checks the size limits and the empty problem, and
checks that device-side problems reach the caller through
fknn_query_tables_noalloc_read_status.  It is collected last so that a
failure here leaves every other test already run.
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


def stream():
    return torch.cuda.current_stream().cuda_stream


def call_noalloc(lib, xyz, steps, neigh, cnt, k, cut_r2=float("inf")):
    n, p = xyz.shape[0], neigh.shape[0]
    idx = torch.full((n, k), -7, dtype=torch.int32, device=DEV)
    dist = torch.full((n, k), float("nan"), dtype=torch.float32, device=DEV)
    rc = lib.fknn_query_tables_noalloc(xyz.data_ptr(), n, steps.data_ptr(), neigh.data_ptr(),
                                       cnt.data_ptr(), p, k, cut_r2, idx.data_ptr(),
                                       dist.data_ptr(), stream())
    return rc, idx, dist


def noalloc_status(lib):
    out = ctypes.c_int(-1)
    rc = lib.fknn_query_tables_noalloc_read_status(ctypes.byref(out), stream())
    assert rc == 0, lib.fknn_error_string(rc)
    return out.value


@pytest.fixture(scope="module")
def lib():
    from flashknn_exprepo_b200 import _lib
    from flashknn_exprepo_b200.build import build
    build()
    return _lib.load()


def test_noalloc_matches_workspace_entry_point_on_consecutive_calls(lib):
    from flashknn_exprepo_b200 import _lib, ops
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
            assert noalloc_status(lib) == 0, case


@pytest.mark.parametrize("what", ["points", "parents"])
def test_noalloc_rejects_problems_beyond_its_scratch(lib, what):
    from flashknn_exprepo_b200 import _lib
    xyz, steps, neigh, cnt, k = tables("uniform_k16")
    n, p = xyz.shape[0], neigh.shape[0]
    if what == "points":
        n = 32769
    else:
        p = 32769
    rc = lib.fknn_query_tables_noalloc(xyz.data_ptr(), n, steps.data_ptr(), neigh.data_ptr(),
                                       cnt.data_ptr(), p, k, float("inf"), None, None, stream())
    assert rc == _lib.FKNN_ERR_SCRATCH_LIMIT
    assert b"scratch" in lib.fknn_error_string(rc)


def test_noalloc_empty_problem_writes_nothing(lib):
    from flashknn_exprepo_b200 import _lib
    rc = lib.fknn_query_tables_noalloc(None, 0, None, None, None, 0, 16, float("inf"), None,
                                       None, stream())
    assert rc == _lib.FKNN_OK, lib.fknn_error_string(rc)
    assert noalloc_status(lib) == 0


def test_noalloc_reports_malformed_tables_then_recovers(lib):
    from flashknn_exprepo_b200 import _lib, ops
    xyz, steps, neigh, cnt, k = tables("uniform_k16")
    bad = neigh.clone()
    busy = torch.nonzero(cnt[:, 27] > 0).flatten()[:5]
    bad[busy, 0] = neigh.shape[0] + 7  # a neighbour row outside the table
    rc, _, _ = call_noalloc(lib, xyz, steps, bad, cnt, k)
    assert rc == _lib.FKNN_OK
    assert noalloc_status(lib) & _lib.DEVICE_BAD_TABLE
    # the next call clears the word and answers as the workspace entry point
    want_idx, want_dist = ops.query_tables(xyz, steps, neigh, cnt, k)
    rc, idx, dist = call_noalloc(lib, xyz, steps, neigh, cnt, k)
    assert rc == _lib.FKNN_OK
    assert noalloc_status(lib) == 0
    assert torch.equal(idx, want_idx)
    assert torch.equal(dist.view(torch.int32), want_dist.view(torch.int32))
