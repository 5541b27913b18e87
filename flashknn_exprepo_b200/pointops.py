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


def knn_query_host(nsample, xyz, offset, idx_out=None, dist_out=None, *, voxel_size,
                   num_down=2, chunks=8, device=None, config=None):
    """Self query of an offset batch held in host memory, answers written to
    host memory: the call for a caller whose points arrive from and whose
    neighbours go back to the CPU.

    The batch is cut into ``chunks`` runs of whole clouds of about equal size
    (8 by default: fewer runs leave more of the first run's upload and query
    outside the overlap, more runs cost more host-side launch work than they
    hide).
    Each run's upload, query and index shift run on the current stream, and
    its download starts on a second stream as soon as the run is done, so the
    device-to-host copy of one run overlaps the upload and query of the next
    (the copies, 8*nsample bytes per point, are the bound on a PCIe host).
    Clouds are independent, so the answer equals one ``knn_query`` over the
    whole batch.  ``xyz`` f32 [n,3] and the outputs should be pinned for the
    copies to be asynchronous; the call returns when the work is queued:
    synchronise the current stream before reading the outputs.
    Returns (idx int32 [n, nsample], dist2 f32 [n, nsample]) on the host.
    """
    dev = torch.device(device) if device is not None else torch.device("cuda",
                                                                       torch.cuda.current_device())
    offset = torch.as_tensor(offset, dtype=torch.int64).cpu()
    n = int(offset[-1]) if offset.numel() else 0
    if idx_out is None:
        idx_out = torch.empty((n, nsample), dtype=torch.int32).pin_memory()
    if dist_out is None:
        dist_out = torch.empty((n, nsample), dtype=torch.float32).pin_memory()
    if n == 0:
        return idx_out, dist_out
    # whole-cloud runs of about n / chunks points
    ends = offset.tolist()
    cuts, target = [0], n / max(1, chunks)
    for c, e in enumerate(ends):
        if e >= target * len(cuts) and c + 1 < len(ends) and len(cuts) < chunks:
            cuts.append(c + 1)
    cuts.append(len(ends))
    # every run's cloud ends relative to its first point, uploaded once from
    # pinned memory (a copy from pageable memory would wait for the stream)
    local = offset.clone()
    for a, b in zip(cuts[:-1], cuts[1:]):
        local[a:b] -= ends[a - 1] if a else 0
    local_dev = local.pin_memory().to(dev, non_blocking=True)
    compute = torch.cuda.current_stream(dev)
    copy = torch.cuda.Stream(dev)
    for a, b in zip(cuts[:-1], cuts[1:]):
        if a == b:
            continue
        start = ends[a - 1] if a else 0
        stop = ends[b - 1]
        x = xyz[start:stop].to(dev, non_blocking=True)
        idx, dist = ops.knn_offsets(x, local_dev[a:b], nsample, voxel_size, num_down,
                                    config=config)
        if start:
            idx += start                               # run-local -> batch indices
        done = torch.cuda.Event()
        done.record(compute)
        copy.wait_event(done)
        with torch.cuda.stream(copy):
            idx_out[start:stop].copy_(idx, non_blocking=True)
            dist_out[start:stop].copy_(dist, non_blocking=True)
        idx.record_stream(copy)
        dist.record_stream(copy)
    compute.wait_stream(copy)
    return idx_out, dist_out
