"""The DeLA neighbour hierarchy on the GPU (drop-in for the reference's
``Networks/hierarchy.py``: ``_voxel_first_cuda`` / ``build_flash_hierarchy``).

Per level: voxel-first subsampling of the previous level (one CUDA call,
``fknn_voxel_first``, and one read-back of the level's size with its status
word), then the grid self query at that level's voxel size
(``fknn_knn_offsets``); at the end, for every level below the first, the
nearest-point map from the full cloud to that level (``fknn_back_query``,
K = 1), whose status words are combined on the device and read once.
Output order and types follow the reference: ``forward + backward`` with
int64 tensors.

The caller's stream runs the chain of voxel-first levels; every level's self
query and every back query only needs that level's points, so each runs on
a side stream (a small pool per device) as soon as its level exists, while
the chain goes on.  The caller's stream waits for all of them before the
function returns, and every tensor handed between streams is recorded on
the stream that uses it, so the caching allocator never reuses its memory
early.
"""
from __future__ import annotations

import math

import torch

from . import _lib, ops


_SIDE: dict = {}
_SIDE_STREAMS = 4


def _side_streams(dev: torch.device) -> list:
    """The side streams of a device (created once, reused by every call)."""
    key = dev.index if dev.index is not None else torch.cuda.current_device()
    pool = _SIDE.get(key)
    if pool is None:
        pool = [torch.cuda.Stream(device=dev) for _ in range(_SIDE_STREAMS)]
        _SIDE[key] = pool
    return pool


def voxel_first(xyz: torch.Tensor, size: float, batch_idx: torch.Tensor | None = None
                ) -> torch.Tensor:
    """Indices (int64, ascending) of one point per occupied voxel of edge
    ``size``: the lowest index of the voxel (Networks/hierarchy.py:23-35)."""
    return ops.voxel_first(xyz.float(), size, batch_idx, validate=True)


def build_flash_hierarchy(metric_xyz: torch.Tensor,
                          voxel_sizes: tuple[float, ...] = (0.06, 0.12, 0.24, 0.48),
                          ks: tuple[int, ...] = (24, 24, 24, 24),
                          alpha: int = 16) -> list[torch.Tensor]:
    """Return the DeLA/DeepLA index hierarchy (Networks/hierarchy.py:38-96):
    [nbr_0, sub_1, nbr_1, ..., sub_L, nbr_L, back_L, ..., back_1] where nbr_l
    is the int64 [n_l, k_l] self-query table of level l (grid kNN with
    parent cell = alpha voxels), sub_l the voxel-first indices of level l in
    level l-1, and back_l maps every input point to its nearest level-l point
    (query cell = 2 x level-l voxel)."""
    exponent = round(math.log2(alpha)) if alpha > 0 else 0
    if alpha < 2 or 2 ** exponent != alpha:
        raise ValueError("alpha must be a power of two")
    if len(voxel_sizes) != len(ks):
        raise ValueError("voxel_sizes and ks must have equal length")
    full_xyz = metric_xyz.float().contiguous()
    current = full_xyz
    dev = full_xyz.device
    main = torch.cuda.current_stream(dev)
    side = _side_streams(dev)
    cumulative = torch.arange(len(full_xyz), device=dev)
    forward: list[torch.Tensor] = []
    levels: list[torch.Tensor] = []
    made_on_side: list[torch.Tensor] = []
    for level, (size, k) in enumerate(zip(voxel_sizes, ks)):
        if level:
            local = voxel_first(current, size)   # reads the level's size back
            current = current[local].contiguous()
            cumulative = cumulative[local]
            forward.append(local)
            levels.append(cumulative)
        s = side[level % len(side)]
        s.wait_stream(main)
        current.record_stream(s)
        with torch.cuda.stream(s):
            offsets = torch.full((1,), len(current), dtype=torch.int64, device=dev)
            idx, _ = ops.knn_offsets(current, offsets, int(k), float(size), exponent)
            nbr = idx.long()
        forward.append(nbr)
        made_on_side.append(nbr)
    backward: list[torch.Tensor] = []
    # every back query ORs its status word into its own flag; the flags are
    # combined on the caller's stream and read once
    flags: list[torch.Tensor] = []
    for j, level in enumerate(range(len(levels) - 1, -1, -1)):
        size = voxel_sizes[level + 1]
        # the streams of the smallest levels first: the first level's large
        # self query keeps its stream busy the longest
        s = side[(len(side) - 1 - j) % len(side)]
        s.wait_stream(main)
        full_xyz.record_stream(s)
        levels[level].record_stream(s)
        with torch.cuda.stream(s):
            flag = torch.zeros(1, dtype=torch.int32, device=dev)
            idx, _, _ = ops.back_query(full_xyz, levels[level], size * 2, 1, status_into=flag)
            back = idx[:, 0]
        flags.append(flag)
        backward.append(back)
        made_on_side.append(back)
    for s in side:
        main.wait_stream(s)
    for t in made_on_side + flags:
        t.record_stream(main)
    bits = 0
    if flags:
        status = flags[0]
        for f in flags[1:]:
            status = status | f
        bits = int(status.item())
    if bits & ~_lib.DEVICE_NO_CANDIDATES:
        raise _lib.FknnError(f"back_query: device reported {_lib.status_text(bits)}")
    if bits & _lib.DEVICE_NO_CANDIDATES:
        raise AssertionError("some query points have no support point in their "
                             "neighbourhood; consider a larger query_grid_size")
    return forward + backward
