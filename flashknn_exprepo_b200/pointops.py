"""Pointcept-style offset-batched kNN with a differentiable distance output.

``knn_query(nsample, xyz, offset, new_xyz=None, new_offset=None)`` follows the
calling convention of Pointcept's ``pointops.knn_query``
(Pointcept/libs/pointops/functions/query.py:7-24): ``offset`` holds the
cumulative end of every cloud.  Differences, by design of this path:
  * the candidates of a query are the points of the 27 grid parent cells
    around it (FlashKNN's neighbourhood), so a voxel size is needed;
  * the distances are *squared* FP32 distances, differentiable with respect
    to ``xyz`` and ``new_xyz`` (a hand-written backward kernel);
  * padding: a self query pads with the point's own index and +inf, a query
    with separate ``new_xyz`` pads with -1 and +inf (Pointcept pads with -1).
"""
from __future__ import annotations

import math

import torch

from . import ops


def default_voxel(xyz, offset, num_down=2):
    """Voxel such that a parent cell spans about two mean point spacings.

    Reads the bounding box back to the host (one synchronisation)."""
    lo = xyz.min(0).values
    hi = xyz.max(0).values
    vol = float(torch.prod(torch.clamp(hi - lo, min=1e-6)).item())
    n = max(int(xyz.shape[0]), 1)
    spacing = (vol / n) ** (1.0 / 3.0)
    return 2.0 * spacing / (1 << num_down)


class KNNQuery(torch.autograd.Function):
    """(idx int32 [m,k], dist2 f32 [m,k]); dist2 is differentiable."""

    @staticmethod
    def forward(ctx, nsample, xyz, offset, new_xyz, new_offset, voxel_size, num_down, cut_r2):
        idx, dist = ops.knn_offsets(xyz, offset, nsample, voxel_size, num_down, new_xyz,
                                    new_offset, cut_r2)
        ctx.mark_non_differentiable(idx)
        ctx.self_query = new_xyz is None
        ctx.save_for_backward(xyz, new_xyz if new_xyz is not None else xyz, idx, dist)
        return idx, dist

    @staticmethod
    def backward(ctx, grad_idx, grad_dist):
        xyz, qxyz, idx, dist = ctx.saved_tensors
        if grad_dist is None:
            return (None,) * 8
        grad_dist = grad_dist.contiguous().float()
        need_p = ctx.needs_input_grad[1]
        need_q = ctx.needs_input_grad[3]
        grad_xyz = grad_new = None
        if ctx.self_query:
            if need_p:
                grad_xyz = torch.zeros_like(xyz, dtype=torch.float32)
                ops.backward(qxyz, xyz, idx, dist, grad_dist, grad_q=grad_xyz, grad_p=grad_xyz,
                             accumulate=True)
        elif need_p or need_q:
            grad_xyz = torch.empty_like(xyz, dtype=torch.float32) if need_p else None
            grad_new = torch.empty_like(qxyz, dtype=torch.float32) if need_q else None
            ops.backward(qxyz, xyz, idx, dist, grad_dist, grad_q=grad_new, grad_p=grad_xyz)
        return None, grad_xyz, None, grad_new, None, None, None, None


def knn_query(nsample, xyz, offset, new_xyz=None, new_offset=None, *, voxel_size=None,
              num_down=2, cut_radius=math.inf):
    """Grid kNN over offset-batched clouds; returns (idx int32, dist2 f32)."""
    if voxel_size is None:
        voxel_size = default_voxel(xyz, offset, num_down)
    if new_xyz is not None and new_offset is None:
        raise ValueError("new_offset is required with new_xyz")
    return KNNQuery.apply(int(nsample), xyz, offset, new_xyz, new_offset, float(voxel_size),
                          int(num_down), float(cut_radius) * float(cut_radius))


def ball_query(nsample, max_radius, min_radius, xyz, offset, new_xyz=None, new_offset=None, *,
               voxel_size=None, num_down=2):
    """Pointcept's ``pointops.ball_query`` calling convention
    (Pointcept/libs/pointops/functions/query.py:73-108) on the grid: the
    nsample nearest points with squared distance below max_radius^2, rows
    ascending, padding (-1, 1e10) before the square root, and returns
    (idx int32 [m, nsample], distance f32 [m, nsample]).

    The default voxel makes a parent cell max_radius wide, so the 27 parent
    cells hold the whole ball and the rows are exact.  Differences from
    Pointcept's brute-force kernel: a ball with more than nsample points
    yields its nsample nearest (Pointcept: a strided subset of them), and
    min_radius must be 0.
    """
    if min_radius != 0:
        raise ValueError("min_radius > 0 is not supported by the grid ball query")
    if not max_radius > 0:
        raise ValueError("max_radius must be positive")
    if voxel_size is None:
        voxel_size = float(max_radius) / (1 << num_down)
    if new_xyz is None or new_offset is None:
        new_xyz, new_offset = None, None
    idx, dist2 = ops.ball_query_offsets(xyz, offset, int(nsample), float(max_radius),
                                        float(voxel_size), int(num_down), new_xyz, new_offset)
    dist2 = torch.where(idx < 0, torch.full_like(dist2, 1e10), dist2)
    return idx, torch.sqrt(dist2)


class Grouping(torch.autograd.Function):
    """Gather of neighbour rows with a deterministic hand-written backward
    (Pointcept/libs/pointops/functions/grouping.py:36-60 semantics)."""

    @staticmethod
    def forward(ctx, idx, feat, xyz, new_xyz, with_xyz):
        idx = idx.to(torch.int32).contiguous()
        out = ops.group_features(feat.float(), idx, xyz, new_xyz, with_xyz)
        ctx.with_xyz = with_xyz
        ctx.self_query = with_xyz and new_xyz is xyz
        ctx.shape = (feat.shape[0], feat.shape[1])
        ctx.save_for_backward(idx)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        (idx,) = ctx.saved_tensors
        n, c = ctx.shape
        grad_out = grad_out.contiguous().float()
        dev = grad_out.device
        need_feat, need_xyz, need_new = ctx.needs_input_grad[1:4]
        if not ctx.with_xyz:
            need_xyz = need_new = False
        grad_feat = torch.empty((n, c), dtype=torch.float32, device=dev)
        grad_xyz = grad_new = None
        if ctx.self_query and (need_xyz or need_new):
            grad_xyz = torch.empty((n, 3), dtype=torch.float32, device=dev)
            ops.group_backward(grad_out, idx, n, c, True, grad_feat, grad_xyz, False, grad_xyz,
                               True)
            return None, grad_feat if need_feat else None, grad_xyz, None, None
        if need_xyz:
            grad_xyz = torch.empty((n, 3), dtype=torch.float32, device=dev)
        if need_new:
            grad_new = torch.empty((idx.shape[0], 3), dtype=torch.float32, device=dev)
        ops.group_backward(grad_out, idx, n, c, ctx.with_xyz, grad_feat, grad_xyz, False,
                           grad_new, False)
        return None, grad_feat if need_feat else None, grad_xyz, grad_new, None


def grouping(idx, feat, xyz, new_xyz=None, with_xyz=False):
    """Pointcept's ``pointops.grouping(idx, feat, xyz, new_xyz, with_xyz)``:
    (m, nsample, c) or, with ``with_xyz``, (m, nsample, 3 + c) whose first
    three channels are the neighbour's offset from the query; idx -1 rows are
    zero."""
    if new_xyz is None:
        new_xyz = xyz
    return Grouping.apply(idx, feat, xyz, new_xyz, bool(with_xyz))


def knn_query_and_group(feat, xyz, offset=None, new_xyz=None, new_offset=None, idx=None,
                        nsample=None, with_xyz=False, *, voxel_size=None, num_down=2):
    """Pointcept's ``pointops.knn_query_and_group``
    (Pointcept/libs/pointops/functions/utils.py:5-18): the grid kNN
    (``knn_query``) unless ``idx`` is given, then ``grouping``.  Returns
    (grouped features, idx)."""
    if idx is None:
        if nsample is None:
            raise ValueError("nsample is required when idx is not given")
        idx, _ = knn_query(nsample, xyz, offset, new_xyz, new_offset, voxel_size=voxel_size,
                           num_down=num_down)
    return grouping(idx, feat, xyz, new_xyz, with_xyz), idx


def ball_query_and_group(feat, xyz, offset=None, new_xyz=None, new_offset=None, idx=None,
                         max_radio=None, min_radio=0, nsample=None, with_xyz=False, *,
                         voxel_size=None, num_down=2):
    """Pointcept's ``pointops.ball_query_and_group`` (utils.py:21-39) on the
    grid ball query."""
    if idx is None:
        if nsample is None or max_radio is None:
            raise ValueError("nsample and max_radio are required when idx is not given")
        idx, _ = ball_query(nsample, max_radio, min_radio, xyz, offset, new_xyz, new_offset,
                            voxel_size=voxel_size, num_down=num_down)
    return grouping(idx, feat, xyz, new_xyz, with_xyz), idx
