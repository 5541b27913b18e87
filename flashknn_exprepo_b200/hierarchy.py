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
"""
from __future__ import annotations

import math

import torch

from . import _lib, ops


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
    cumulative = torch.arange(len(full_xyz), device=dev)
    forward: list[torch.Tensor] = []
    levels: list[torch.Tensor] = []
    for level, (size, k) in enumerate(zip(voxel_sizes, ks)):
        if level:
            local = voxel_first(current, size)
            current = current[local].contiguous()
            cumulative = cumulative[local]
            forward.append(local)
            levels.append(cumulative)
        offsets = torch.full((1,), len(current), dtype=torch.int64, device=dev)  # no host copy
        idx, _ = ops.knn_offsets(current, offsets, int(k), float(size), exponent)
        forward.append(idx.long())
    backward: list[torch.Tensor] = []
    # the back queries' status words are OR-ed on the device and read once
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    for level in range(len(levels) - 1, -1, -1):
        size = voxel_sizes[level + 1]
        idx, _, _ = ops.back_query(full_xyz, levels[level], size * 2, 1, status_into=status)
        backward.append(idx[:, 0])
    bits = int(status.item()) if levels else 0
    if bits & ~_lib.DEVICE_NO_CANDIDATES:
        raise _lib.FknnError(f"back_query: device reported {_lib.status_text(bits)}")
    if bits & _lib.DEVICE_NO_CANDIDATES:
        raise AssertionError("some query points have no support point in their "
                             "neighbourhood; consider a larger query_grid_size")
    return forward + backward
