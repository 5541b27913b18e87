"""Drop-in for the reference's ``AdaptiveNeighborhoodFlashKNN``
(FlashKNN/functions/adaptive_octree.py:491-612).

Each point takes its K nearest neighbours among the points of the 27 nodes
around its own node on one level of a Morton octree; the level is chosen per
point, coarse to fine, so that the candidate count lands between
``min_candidates_factor * K`` and ``max_candidates_factor * K`` where it can
(sparse far-field LiDAR points get coarse levels, dense ones fine levels).
Everything -- octree levels, selection, query groups and the top-K -- runs
on the GPU in one C-ABI call (``fknn_adaptive_query``) that never copies
coordinates per level.
"""
from __future__ import annotations

import math

import torch

from . import _lib, ops


class AdaptiveNeighborhoodFlashKNN:
    """FlashKNN with an independently selected octree level per query point."""

    def __init__(self, num_nbr: int = 32, min_candidates_factor: int = 2,
                 max_candidates_factor: int = 8):
        self.num_nbr = num_nbr
        self.min_candidates_factor = min_candidates_factor
        self.max_candidates_factor = max_candidates_factor
        self.last_levels = None
        self._stats = None

    @staticmethod
    def _validate(grid_coord, batch_idx):
        # the reference's checks (adaptive_octree.py:113-126)
        if not grid_coord.is_cuda or not batch_idx.is_cuda:
            raise ValueError("adaptive octree inputs must be CUDA tensors")
        if grid_coord.dtype != torch.int64 or batch_idx.dtype != torch.int64:
            raise ValueError("grid_coord and batch_idx must use torch.int64")
        if grid_coord.ndim != 2 or grid_coord.shape[1] != 3:
            raise ValueError("grid_coord must have shape [N, 3]")
        if batch_idx.ndim != 1 or batch_idx.shape[0] != grid_coord.shape[0]:
            raise ValueError("batch_idx must have shape [N]")
        if grid_coord.shape[0] == 0:
            raise ValueError("cannot construct an octree for an empty point cloud")

    @torch.no_grad()
    def query(self, grid_coord: torch.Tensor, batch_idx: torch.Tensor,
              xyz: torch.Tensor | None = None, *, max_shift: int | None = None,
              batch_for_prune: int = 1, cut_radius: float = math.inf,
              return_distances: bool = False):
        """int64 neighbour indices [N, K] (and FP32 squared distances with
        ``return_distances``), in input numbering and order.  ``xyz=None``
        measures distances on the grid coordinates translated to each batch's
        minimum, as the reference does.  ``batch_for_prune`` is accepted and
        ignored, as by the reference kernel."""
        del batch_for_prune
        self._validate(grid_coord, batch_idx)
        k = self.num_nbr
        if k <= 0:
            raise ValueError("k must be positive")
        if self.min_candidates_factor < 1:
            raise ValueError("min_candidates_factor must be at least one")
        if self.max_candidates_factor < self.min_candidates_factor:
            raise ValueError("max_candidates_factor must not be smaller than min")
        if max_shift is not None and not 0 <= max_shift <= 16:
            raise ValueError("max_shift must lie in [0, 16]")
        n = grid_coord.shape[0]
        if n < k:
            raise ValueError(f"point cloud contains {n} points, fewer than k={k}")
        idx, dist, levels = ops.adaptive_query(
            grid_coord, batch_idx, k, xyz=xyz, min_factor=self.min_candidates_factor,
            max_factor=self.max_candidates_factor, max_shift=max_shift,
            cut_r2=float(cut_radius) * float(cut_radius), want_levels=True)
        status = _lib.read_status(_lib.WORKSPACE.get(0, grid_coord.device))
        if status & _lib.DEVICE_BATCH_RANGE:
            raise ValueError("batch indices must lie in [0, 32768)")
        if status & _lib.DEVICE_COORD_RANGE:
            raise ValueError("each batch's coordinate span must be smaller than 65536")
        if status:
            _lib.raise_on_status(_lib.WORKSPACE.get(0, grid_coord.device), "adaptive_query")
        self.last_levels = levels
        self._stats = None
        if return_distances:
            return idx, dist
        return idx

    @property
    def last_stats(self) -> dict:
        """Level statistics of the last query (computed on first access)."""
        if self._stats is None and self.last_levels is not None:
            counts = torch.bincount(self.last_levels.long(), minlength=17).tolist()
            self._stats = {
                "k": self.num_nbr,
                "min_candidates_factor": self.min_candidates_factor,
                "max_candidates_factor": self.max_candidates_factor,
                "selected_level_points": {lv: c for lv, c in enumerate(counts) if c},
                "query_kernel_launches": 1,
            }
        return self._stats or {}
