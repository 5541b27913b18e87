"""The reference's compiled kernel module ``FlashKNN.CuFun`` on this library.

FlashKNN/functions/FlashKnnWrapper.py:6-19 imports twelve names from the
pybind11 module built from FlashKNN/csrc/api.cpp:7-20.  This module exports
the same twelve names with the same positional arguments, the same tensor
layouts and the same in-place outputs, and runs each through the C ABI
(libfknn.so), so the unchanged wrapper works when a maintainer makes it
import them from here (for example a ``FlashKNN/functions/CuFun.py`` holding
``from flashknn_exprepo_b200.cufun import *``).

Mapping (all launches on the current stream; no device-wide synchronise):

* ``FlashKNN_Query_Dynamic_Load`` and its ablation variants
  (``_Ablation``, ``_Thread_Group``, ``FlashKNN_Query_GMPS``,
  ``FlashKNN_Query_SMSS``, flash_knn_query.h:144-181,235-257), which compute
  the same top-K over the same tables: ``fknn_query_tables``;
* ``FlashKNN_Selected_Query_DL`` (:206-218): ``fknn_selected_query_tables``;
* ``FlashKNN_Query_GM`` (:220-233) and the back-query kernels
  ``FlashKNN_Nearest_Back_Query_DL`` / ``FlashKNN_Back_Query_DL``
  (:183-204): ``fknn_general_query_tables``;
* ``FlashKNN_Morton_Encode`` / ``FlashKNN_Morton_Neighbor_Keys``
  (flash_knn_construction.h:7-13): ``fknn_morton_encode`` /
  ``fknn_morton_neighbor_keys``;
* ``get_cuda_shared_mem``: the device's opt-in shared memory per block.

Differences a caller sees: rows are ascending by (distance, index) (the
reference's back-query kernels leave K > 1 rows in heap order), the nearest
back query pads a point without candidates with (0, +inf) instead of
(0, -1) (the wrapper asserts that this never happens), and failures raise
:class:`FknnError` (a RuntimeError) instead of throwing
``cudaErrorNotYetImplemented``.
"""
from __future__ import annotations

import math

import torch

from . import _lib, ops
from ._lib import check, ptr, stream_handle

__all__ = [
    "FlashKNN_Back_Query_DL", "FlashKNN_Morton_Encode", "FlashKNN_Morton_Neighbor_Keys",
    "FlashKNN_Nearest_Back_Query_DL", "FlashKNN_Query_Dynamic_Load",
    "FlashKNN_Query_Dynamic_Load_Ablation", "FlashKNN_Query_Dynamic_Load_Thread_Group",
    "FlashKNN_Query_GM", "FlashKNN_Query_GMPS", "FlashKNN_Query_SMSS",
    "FlashKNN_Selected_Query_DL", "get_cuda_shared_mem",
]


def _out(t: torch.Tensor, dtype, name: str) -> torch.Tensor:
    """The reference writes into the caller's tensor: it must already be a
    contiguous CUDA tensor of the right type."""
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == dtype and t.is_contiguous()):
        raise _lib.FknnError(f"{name} must be a contiguous CUDA {dtype} tensor")
    return t


def _in(t: torch.Tensor, dtype, name: str) -> torch.Tensor:
    if not (isinstance(t, torch.Tensor) and t.is_cuda):
        raise _lib.FknnError(f"{name} must be a CUDA tensor")
    return t.to(dtype).contiguous()


def get_cuda_shared_mem() -> int:
    """Opt-in shared memory per block of the current device, in bytes."""
    dev = torch.cuda.current_device()
    return int(torch.cuda.get_device_properties(dev).shared_memory_per_block_optin)


def FlashKNN_Query_Dynamic_Load(GridCoord, Parent2Child, ParentNeigh, CumCntInNeigh, K, Indices,
                                Dis, batch_for_prune=8, cut_radiu2=math.inf):
    lib = _lib.load()
    xyz = _in(GridCoord, torch.float32, "GridCoord")
    steps = _in(Parent2Child, torch.int32, "Parent2Child")
    neigh = _in(ParentNeigh, torch.int32, "ParentNeigh")
    cnt = _in(CumCntInNeigh, torch.int32, "CumCntInNeigh")
    idx = _out(Indices, torch.int32, "Indices")
    dis = _out(Dis, torch.float32, "Dis")
    n, p = xyz.shape[0], neigh.shape[0]
    if idx.numel() < n * K or dis.numel() < n * K:
        raise _lib.FknnError("Indices and Dis must hold N x K entries")
    ws = _lib.WORKSPACE.get(lib.fknn_tables_workspace_bytes(n, n, p), xyz.device)
    check(lib.fknn_query_tables(ptr(xyz), n, ptr(steps), ptr(neigh), ptr(cnt), p, int(K),
                                float(cut_radiu2), ptr(idx), ptr(dis), ptr(ws), ws.numel(), None,
                                stream_handle(xyz.device)), "FlashKNN_Query_Dynamic_Load")


def FlashKNN_Query_Dynamic_Load_Ablation(GridCoord, Parent2Child, ParentNeigh, CumCntInNeigh, K,
                                         Indices, Dis, batch_for_prune, cut_radiu2,
                                         candidate_in_shared, enable_skip):
    """Candidate placement / skip ablation: the same top-K."""
    FlashKNN_Query_Dynamic_Load(GridCoord, Parent2Child, ParentNeigh, CumCntInNeigh, K, Indices,
                                Dis, batch_for_prune, cut_radiu2)


def FlashKNN_Query_Dynamic_Load_Thread_Group(GridCoord, Parent2Child, ParentNeigh, CumCntInNeigh,
                                             K, Indices, Dis, batch_for_prune, cut_radiu2,
                                             thread_group_size):
    """Fixed thread-group ablation: the same top-K."""
    FlashKNN_Query_Dynamic_Load(GridCoord, Parent2Child, ParentNeigh, CumCntInNeigh, K, Indices,
                                Dis, batch_for_prune, cut_radiu2)


def FlashKNN_Query_GMPS(GridCoord, Parent2Child, ParentNeigh, CumCntInNeigh, K, Indices, Dis,
                        batch_for_prune, cut_radiu2):
    """Global-memory / parallel-sort ablation: the same top-K."""
    FlashKNN_Query_Dynamic_Load(GridCoord, Parent2Child, ParentNeigh, CumCntInNeigh, K, Indices,
                                Dis, batch_for_prune, cut_radiu2)


def FlashKNN_Query_SMSS(GridCoord, Parent2Child, ParentNeigh, CumCntInNeigh, K, Indices, Dis,
                        batch_for_prune, cut_radiu2):
    """Shared-memory / serial-sort ablation: the same top-K."""
    FlashKNN_Query_Dynamic_Load(GridCoord, Parent2Child, ParentNeigh, CumCntInNeigh, K, Indices,
                                Dis, batch_for_prune, cut_radiu2)


def FlashKNN_Selected_Query_DL(GridCoord, Queryindex, Parent2Child, Parent2ChildQuery,
                               ParentNeigh, CumCntInNeigh, K, Indices, Dis, batch_for_prune,
                               cut_radiu2):
    lib = _lib.load()
    xyz = _in(GridCoord, torch.float32, "GridCoord")
    qidx = _in(Queryindex, torch.int32, "Queryindex")
    steps = _in(Parent2Child, torch.int32, "Parent2Child")
    steps_q = _in(Parent2ChildQuery, torch.int32, "Parent2ChildQuery")
    neigh = _in(ParentNeigh, torch.int32, "ParentNeigh")
    cnt = _in(CumCntInNeigh, torch.int32, "CumCntInNeigh")
    idx = _out(Indices, torch.int32, "Indices")
    dis = _out(Dis, torch.float32, "Dis")
    n, m, p = xyz.shape[0], qidx.numel(), neigh.shape[0]
    if idx.numel() < m * K or dis.numel() < m * K:
        raise _lib.FknnError("Indices and Dis must hold M x K entries")
    ws = _lib.WORKSPACE.get(lib.fknn_tables_workspace_bytes(n, m, p), xyz.device)
    check(lib.fknn_selected_query_tables(ptr(xyz), n, ptr(qidx), m, ptr(steps), ptr(steps_q),
                                         ptr(neigh), ptr(cnt), p, int(K), float(cut_radiu2),
                                         ptr(idx), ptr(dis), ptr(ws), ws.numel(), None,
                                         stream_handle(xyz.device)),
          "FlashKNN_Selected_Query_DL")


def _general(name, xyz_s, xyz_q, steps_s, steps_q, pad, neigh, cnt, k, idx_out, dis_out, cut_r2):
    lib = _lib.load()
    xs = _in(xyz_s, torch.float32, "support xyz")
    xq = _in(xyz_q, torch.float32, "query xyz")
    ss = _in(steps_s, torch.int32, "support Parent2Child")
    sq = _in(steps_q, torch.int32, "query Parent2Child")
    nb = _in(neigh, torch.int32, "ParentNeigh")
    cn = _in(cnt, torch.int32, "CumCntInNeigh")
    pd = None if pad is None else _in(pad, torch.int32, "QueryIndex")
    idx = _out(idx_out, torch.int32, "Indices")
    dis = _out(dis_out, torch.float32, "Dis")
    n, m, p = xs.shape[0], xq.shape[0], nb.shape[0]
    if idx.numel() < m * k or dis.numel() < m * k:
        raise _lib.FknnError("Indices and Dis must hold M x K entries")
    ws = _lib.WORKSPACE.get(lib.fknn_tables_workspace_bytes(n, m, p), xs.device)
    check(lib.fknn_general_query_tables(ptr(xs), n, ptr(xq), m, ptr(pd), ptr(ss), ptr(sq),
                                        ptr(nb), ptr(cn), p, int(k), float(cut_r2), ptr(idx),
                                        ptr(dis), ptr(ws), ws.numel(), None,
                                        stream_handle(xs.device)), name)


def FlashKNN_Query_GM(xyz_Support, xyz_Query, Parent2Child_Support, Parent2Child_Query,
                      QueryIndex, Query2Parent, ParentNeigh, CumCntInNeigh, Indices_out, Dis_out,
                      num_nbr, cut_radiu2=math.inf):
    """Query2Parent is implied by Parent2Child_Query and not read."""
    _general("FlashKNN_Query_GM", xyz_Support, xyz_Query, Parent2Child_Support,
             Parent2Child_Query, QueryIndex, ParentNeigh, CumCntInNeigh, num_nbr, Indices_out,
             Dis_out, cut_radiu2)


def FlashKNN_Nearest_Back_Query_DL(xyz_H, xyz_L, Parent2Child_H, Parent2Child_L, ParentNeigh,
                                   CumCntInNeigh_L, Indices, Dis_out):
    pad = torch.zeros(xyz_H.shape[0], dtype=torch.int32, device=xyz_H.device)
    _general("FlashKNN_Nearest_Back_Query_DL", xyz_L, xyz_H, Parent2Child_L, Parent2Child_H, pad,
             ParentNeigh, CumCntInNeigh_L, 1, Indices, Dis_out, math.inf)


def FlashKNN_Back_Query_DL(xyz_H, xyz_L, Parent2Child_H, Parent2Child_L, ParentNeigh,
                           CumCntInNeigh_L, num_nbr, Indices, Dis_out):
    _general("FlashKNN_Back_Query_DL", xyz_L, xyz_H, Parent2Child_L, Parent2Child_H, None,
             ParentNeigh, CumCntInNeigh_L, num_nbr, Indices, Dis_out, math.inf)


def FlashKNN_Morton_Encode(grid_coord, batch):
    return ops.morton_encode(grid_coord, batch)


def FlashKNN_Morton_Neighbor_Keys(grid_down, parent_batch):
    return ops.morton_neighbor_keys(grid_down, parent_batch)
