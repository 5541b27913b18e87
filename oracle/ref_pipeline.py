"""The reference's per-cloud query pipeline on the GPU -- TEST/BENCH ONLY.

Restates the fused-construction branch of ``FlashKNN.query``
(FlashKNN/functions/FlashKnnWrapper.py:220-430) step by step with the same
ATen calls, and runs the reference's own kernels compiled for sm_100a
(``oracle.ref_kernels``: FlashKNN_Morton_Encode, FlashKNN_Morton_Neighbor_Keys,
FlashKNN_Query_Dynamic_Load).  Used as the "plain per-cloud kernel" baseline
of the benchmark's reference arm and by the parity tests; never by the
product.
"""
from __future__ import annotations

import math

import torch
import torch.nn.functional as F


def reference_query(cufun, grid_coord, batch_idx, xyz, k, num_down=2, cut_radius=math.inf):
    """Returns (int64 [N,K] original indices, f32 [N,K] distances in sorted
    order remapped like the indices)."""
    t = reference_tables(cufun, grid_coord, batch_idx, xyz, num_down)
    out_indices = torch.zeros((len(grid_coord), k), device=grid_coord.device, dtype=torch.int32)
    out_dis = torch.zeros((len(grid_coord), k), device=grid_coord.device, dtype=torch.float32)
    cufun.FlashKNN_Query_Dynamic_Load(t["xyz_sorted"], t["steps"], t["neigh"], t["cnt"], k,
                                      out_indices, out_dis, 1, cut_radius * cut_radius)
    order, inverse_order = t["order"], t["inverse_order"]
    out = order[out_indices.long()[inverse_order]]
    torch.cuda.synchronize()
    return out, out_dis[inverse_order]


def reference_tables(cufun, grid_coord, batch_idx, xyz, num_down=2):
    """The tables FlashKNN.query hands its kernel (FlashKnnWrapper.py:220-365):
    xyz_sorted f32 [N,3], steps / neigh / cnt int32, plus order and
    inverse_order (int64) for the remap."""
    device = grid_coord.device
    key = cufun.FlashKNN_Morton_Encode(grid_coord.contiguous(), batch_idx.contiguous())
    order = torch.argsort(key)
    key = key[order]
    grid_coord = grid_coord[order]
    inverse_order = torch.empty(len(grid_coord), device=device, dtype=torch.long)
    inverse_order[order] = torch.arange(len(grid_coord), device=device, dtype=torch.long)
    key_down = key >> (3 * num_down)
    key_down_unique, count = torch.unique_consecutive(key_down, return_counts=True)
    steps = F.pad(torch.cumsum(count, dim=0), (1, 0))
    parent_starts = steps[: len(key_down_unique)]
    grid_coord_down = (grid_coord[parent_starts] >> num_down).contiguous()
    parent_batch = batch_idx[order[parent_starts]].contiguous()
    key_down_nbr = cufun.FlashKNN_Morton_Neighbor_Keys(grid_coord_down, parent_batch)
    parent_keys = key_down_nbr[::27].contiguous()
    positions = torch.searchsorted(parent_keys, key_down_nbr)
    safe_positions = positions.clamp_max(len(parent_keys) - 1)
    present = (positions < len(parent_keys)) & (parent_keys[safe_positions] == key_down_nbr)
    neigh = torch.where(present, safe_positions, -1).reshape(-1, 27)
    cnt_in_neigh = F.pad(torch.cumsum(F.pad(count, (0, 1))[neigh], dim=1), [1, 0])
    xyz_sorted = xyz[order].float().contiguous()
    return {"xyz_sorted": xyz_sorted, "steps": steps.int(), "neigh": neigh.int(),
            "cnt": cnt_in_neigh.int(), "order": order, "inverse_order": inverse_order}


def reference_back_query(cufun, xyz, sel_indices, query_grid_size, batch_idx, k):
    """FlashKNN.back_query's fused branch (FlashKnnWrapper.py:459-585) with
    the reference kernels FlashKNN_Nearest_Back_Query_DL (k == 1) and
    FlashKNN_Back_Query_DL (k > 1).  Returns (int64 [N,K] positions in
    sel_indices, f32 [N,K] distances); rows in the kernel's heap order.

    Refuses k > 32: for 33 <= k <= 64 the reference launcher instantiates
    FlashKNN_Back_Query_DL_kernel<float, 4, 5>, whose per-thread candidate
    arrays hold 1 << 5 = 32 entries (flash_knn_query_dynamic_load.cu:1089-1090
    and the launcher's bit_len_K == 6 branch), so it would write past them."""
    if k > 32:
        raise ValueError("the reference back-query kernel overruns its 32-entry list for k > 32")
    device = xyz.device
    grid_coord = (xyz / query_grid_size).long()
    key_h = cufun.FlashKNN_Morton_Encode(grid_coord.contiguous(), batch_idx.contiguous())
    order_h = key_h.argsort()
    inverse_order = torch.empty(len(order_h), device=device, dtype=torch.long)
    inverse_order[order_h] = torch.arange(len(order_h), device=device, dtype=torch.long)
    key_l = key_h[sel_indices]
    order_l = key_l.argsort()
    xyz_l = xyz[sel_indices][order_l]
    key_h = key_h[order_h]
    key_unique_h, child_to_parent, count_h = torch.unique_consecutive(
        key_h, return_inverse=True, return_counts=True)
    steps_h = F.pad(torch.cumsum(count_h, dim=0), (1, 0))
    xyz_h = xyz[order_h]
    count_l = torch.zeros_like(count_h).scatter_add(
        0, child_to_parent[inverse_order[sel_indices]], torch.ones_like(sel_indices))
    steps_l = F.pad(torch.cumsum(count_l, dim=0), (1, 0))
    parent_starts = steps_h[: len(key_unique_h)]
    grid_coord_down = grid_coord[order_h[parent_starts]].contiguous()
    parent_batch = batch_idx[order_h[parent_starts]].contiguous()
    key_down_nbr = cufun.FlashKNN_Morton_Neighbor_Keys(grid_coord_down, parent_batch)
    parent_keys = key_down_nbr[::27].contiguous()
    positions = torch.searchsorted(parent_keys, key_down_nbr)
    safe_positions = positions.clamp_max(len(parent_keys) - 1)
    present = (positions < len(parent_keys)) & (parent_keys[safe_positions] == key_down_nbr)
    neigh = torch.where(present, safe_positions, -1).reshape(-1, 27)
    cnt = F.pad(torch.cumsum(F.pad(count_l, (0, 1))[neigh], dim=1), [1, 0])
    if not bool((cnt[:, -1] != 0).all()):
        raise AssertionError("a query cell has no subset point in its neighbourhood")
    out_indices = torch.zeros((len(grid_coord), k), device=device, dtype=torch.int32)
    out_dis = torch.zeros((len(grid_coord), k), device=device, dtype=torch.float32)
    args = (xyz_h.float().contiguous(), xyz_l.float().contiguous(), steps_h.int(), steps_l.int(),
            neigh.int(), cnt.int())
    if k == 1:
        cufun.FlashKNN_Nearest_Back_Query_DL(*args, out_indices, out_dis)
    else:
        cufun.FlashKNN_Back_Query_DL(*args, k, out_indices, out_dis)
    torch.cuda.synchronize()
    out = order_l[out_indices.long()[inverse_order]]
    return out, out_dis[inverse_order]
