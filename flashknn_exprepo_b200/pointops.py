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
