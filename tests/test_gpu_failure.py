"""Failure detection without a GPU fault.

Device-side problems end the launch early or skip the bad data, set a bit in
the workspace's status word and leave the context usable; the host reads the
word (fknn_read_status) and raises.  Here: a stalled bounded wait (the
self-test arms a barrier that nothing completes), and reference tables that
name rows outside the point array or disagree with each other.  After each
case an ordinary query must still run and match the oracle.
"""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.conftest import GOLDEN

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


def tables():
    z = np.load(os.path.join(GOLDEN, "tables_uniform_k16.npz"))
    return (z["ref_xyz_sorted"].astype(np.float32), z["ref_steps"].astype(np.int32),
            z["ref_neigh"].astype(np.int32), z["ref_cnt"].astype(np.int32), int(z["k"]))


def still_works(fk):
    xyz, steps, neigh, cnt, k = tables()
    gi, gd = fk.ops.query_tables(T(xyz), T(steps), T(neigh), T(cnt), k, validate=True)
    oi, od = O.query_tables(xyz, steps, neigh, cnt, k)
    assert np.array_equal(gi.cpu().numpy(), oi)
    assert np.array_equal(gd.cpu().numpy().view(np.uint32), od.view(np.uint32))


def test_stalled_wait_gives_up_and_is_reported(fk):
    from flashknn_exprepo_b200 import _lib
    lib = _lib.load()
    ws = torch.empty(4096, dtype=torch.uint8, device=DEV)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(lib.fknn_selftest_bounded_wait(_lib.ptr(ws), ws.numel(), 4096, stream),
               "fknn_selftest_bounded_wait")
    assert _lib.read_status(ws) & _lib.DEVICE_TIMEOUT
    assert lib.fknn_selftest_bounded_wait(_lib.ptr(ws), ws.numel(), 0, stream) == _lib.FKNN_ERR_ARG
    still_works(fk)


@pytest.mark.parametrize("fault", ["neigh_out_of_range", "cnt_decreasing", "steps_beyond_points",
                                   "steps_negative"])
def test_malformed_tables_are_reported(fk, fault):
    xyz, steps, neigh, cnt, k = tables()
    p, n = neigh.shape[0], len(xyz)
    neigh, cnt, steps = neigh.copy(), cnt.copy(), steps.copy()
    busy = np.nonzero(cnt[:, 27] > 0)[0][:5]
    if fault == "neigh_out_of_range":
        neigh[busy, 0] = p + 7
    elif fault == "cnt_decreasing":
        cnt[busy, 5] = cnt[busy, 4] - 3
    elif fault == "steps_beyond_points":
        steps[busy + 1] = n + 100
    else:
        steps[busy] = -50
    with pytest.raises(fk.FknnError, match="table"):
        fk.ops.query_tables(T(xyz), T(steps), T(neigh), T(cnt), k, validate=True)
    still_works(fk)


def test_selected_query_index_out_of_range(fk):
    z = np.load(os.path.join(GOLDEN, "tables_uniform_selected_k16.npz"))
    qidx = z["ref_qindex"].astype(np.int32).copy()
    qidx[3] = len(z["ref_xyz_sorted"]) + 5
    with pytest.raises(fk.FknnError, match="table"):
        fk.ops.selected_query_tables(T(z["ref_xyz_sorted"].astype(np.float32)), T(qidx),
                                     T(z["ref_steps"].astype(np.int32)),
                                     T(z["ref_steps_query"].astype(np.int32)),
                                     T(z["ref_neigh"].astype(np.int32)),
                                     T(z["ref_cnt"].astype(np.int32)), int(z["k"]),
                                     validate=True)
    still_works(fk)
