"""GPU: the CuFun-compatible module (flashknn_exprepo_b200.cufun) under the
reference wrapper's own call sequence.

oracle/ref_pipeline.py restates the fused branches of FlashKNN.query and
FlashKNN.back_query (FlashKNN/functions/FlashKnnWrapper.py:220-430, 459-585)
call by call -- the same ATen construction and the same CuFun calls in the
same order with the same arguments.  Here it is driven by our module in
place of the compiled reference module: the answers must equal this
library's fused entry points (bit-identical distances; indices equal up to
ties at the K-th distance, which the table path breaks by sorted position
and the fused path by point index) and the oracle.  The reference checkout
itself is not available where these tests run; tests/test_cufun_cpu.py
checks against it that the module exports what the wrapper imports.
"""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.conftest import GOLDEN
from tests.test_gpu_reference_parity import compare_up_to_kth_ties, grid_of
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


def wrapper_query_on_shim(xyz, voxel, k, num_down=2, batch=None):
    from flashknn_exprepo_b200 import cufun
    from oracle import ref_pipeline
    grid = T(grid_of(xyz, voxel))
    b = T(batch) if batch is not None else torch.zeros(len(xyz), dtype=torch.int64, device=DEV)
    i, d = ref_pipeline.reference_query(cufun, grid, b, T(xyz), k, num_down)
    return grid, b, i.cpu().numpy(), d.cpu().numpy()


@pytest.mark.parametrize("case", ["cube", "uniform_k16", "dense_multibatch_k64",
                                  "two_clouds_negative_k8"])
def test_wrapper_query_sequence_on_the_shim(fk, case):
    from flashknn_exprepo_b200 import synthetic as S
    if case == "cube":
        xyz, k, nd, batch = S.uniform_cube(), 16, 2, None
        grid, b, ii, dd = wrapper_query_on_shim(xyz, S.C1_VOXEL, k, nd)
    else:
        z = np.load(os.path.join(GOLDEN, f"tables_{case}.npz"))
        xyz, k, nd, batch = z["xyz"], int(z["k"]), int(z["num_down"]), z["batch"]
        from flashknn_exprepo_b200 import cufun
        from oracle import ref_pipeline
        b = T(batch)
        i, d = ref_pipeline.reference_query(cufun, T(z["grid"]), b, T(xyz), k, nd)
        grid, ii, dd = T(z["grid"]), i.cpu().numpy(), d.cpu().numpy()
    gi, gd = fk.FlashKNN(num_nbr=k, num_down=nd).query(grid, b if batch is not None else None,
                                                     T(xyz), return_distances=True)
    compare_up_to_kth_ties(gi.cpu().numpy().astype(np.int64), gd.cpu().numpy(), ii, dd)
    oi, od = O.knn_general(xyz, grid.cpu().numpy(), None if batch is None else batch, xyz,
                           grid.cpu().numpy(), None if batch is None else batch, nd, k,
                           pad=np.arange(len(xyz)))
    compare_up_to_kth_ties(oi.astype(np.int64), od, ii, dd)


@pytest.mark.parametrize("case", back_cases())
def test_wrapper_back_query_sequence_on_the_shim(fk, case):
    """FlashKNN_Nearest_Back_Query_DL / FlashKNN_Back_Query_DL through
    fknn_general_query_tables, under the wrapper's own back-query tables."""
    from flashknn_exprepo_b200 import cufun
    from oracle import ref_pipeline
    z = np.load(os.path.join(GOLDEN, f"back_{case}.npz"))
    k = int(z["k"])
    n = len(z["xyz"])
    batch = z["batch"] if len(z["batch"]) else np.zeros(n, np.int64)
    size = float(z["query_grid_size"])
    si, sd = ref_pipeline.reference_back_query(cufun, T(z["xyz"]), T(z["sel"]), size, T(batch), k)
    oi, od, _ = O.back_query(z["xyz"], z["sel"], size, k, batch)
    assert same_up_to_kth_ties(oi.astype(np.int64), od, si.cpu().numpy(), sd.cpu().numpy())


def test_query_gm_equals_dynamic_load_on_the_same_tables(fk):
    """FlashKNN_Query_GM as the wrapper calls it for a self query
    (FlashKnnWrapper.py:401-414: support = queries, QueryIndex = arange)
    answers as FlashKNN_Query_Dynamic_Load does."""
    from flashknn_exprepo_b200 import cufun
    z = np.load(os.path.join(GOLDEN, "tables_uniform_k16.npz"))
    xyz, steps, neigh, cnt = (T(z["ref_xyz_sorted"]), T(z["ref_steps"]), T(z["ref_neigh"]),
                              T(z["ref_cnt"]))
    k, n = int(z["k"]), len(z["ref_xyz_sorted"])
    i1 = torch.zeros((n, k), dtype=torch.int32, device=DEV)
    d1 = torch.zeros((n, k), dtype=torch.float32, device=DEV)
    cufun.FlashKNN_Query_Dynamic_Load(xyz, steps, neigh, cnt, k, i1, d1, 1, float("inf"))
    i2 = torch.zeros_like(i1)
    d2 = torch.zeros_like(d1)
    parent = torch.repeat_interleave(torch.arange(neigh.shape[0], device=DEV),
                                     (steps[1:] - steps[:-1]).long())
    cufun.FlashKNN_Query_GM(xyz, xyz, steps, steps, torch.arange(n, device=DEV), parent, neigh,
                            cnt, i2, d2, k, float("inf"))
    assert torch.equal(i1, i2) and torch.equal(d1.view(torch.int32), d2.view(torch.int32))
    oi, od = O.query_tables(z["ref_xyz_sorted"], z["ref_steps"], z["ref_neigh"], z["ref_cnt"], k)
    assert np.array_equal(i1.cpu().numpy(), oi)
    assert np.array_equal(d1.cpu().numpy().view(np.uint32), od.view(np.uint32))


def test_general_tables_pad_rules(fk):
    """A query whose parent has no candidates is padded with its pad index
    (or -1 without one) and +inf."""
    sx = T(np.array([[0.1, 0.1, 0.1], [0.2, 0.1, 0.1]], np.float32))
    qx = T(np.array([[0.12, 0.1, 0.1], [5.0, 5.0, 5.0]], np.float32))  # nearer point 0
    steps = T(np.array([0, 2, 2], np.int32))          # parent 1 holds no support point
    steps_q = T(np.array([0, 1, 2], np.int32))
    neigh = np.full((2, 27), -1, np.int32)
    neigh[0, 0], neigh[1, 0] = 0, 1
    cnt = np.zeros((2, 28), np.int32)
    cnt[0, 1:] = 2
    i, d = fk.ops.general_query_tables(sx, qx, steps, steps_q, T(neigh), T(cnt), 2,
                                       validate=True)
    assert i.cpu().tolist() == [[0, 1], [-1, -1]]
    assert np.isinf(d.cpu().numpy()[1]).all()
    i, _ = fk.ops.general_query_tables(sx, qx, steps, steps_q, T(neigh), T(cnt), 3,
                                       pad_index=T(np.array([7, 9], np.int32)))
    assert i.cpu().tolist() == [[0, 1, 7], [9, 9, 9]]
