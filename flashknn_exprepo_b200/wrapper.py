"""Drop-in for the reference's ``FlashKNN`` class
(FlashKNN/functions/FlashKnnWrapper.py:22-849).

Same constructor, same ``query`` / ``selected_query`` signatures and the same
return values: int64 neighbour indices in the caller's point numbering, rows
in the caller's query order.  Behind them one C-ABI call runs the whole
construction + query on the device (no host synchronisation), instead of the
reference's ~15 ATen calls, two host syncs and a device-wide synchronise.

The reference's ablation switches (``memory_mode`` GM, ``sorting_mode`` SS,
``candidate_mode`` shared, ``enable_skip`` False, ``thread_group_size``)
select alternative reference kernels that compute the same exact top-K over
the same candidates.  They are validated exactly as the reference validates
them (FlashKnnWrapper.py:193-219) and then served by the one B200 kernel; the
result is the same set of neighbours.
"""
from __future__ import annotations

import math
import time

import numpy as np
import torch

from . import ops
from ._lib import FknnError


class FlashKNN:
    def __init__(self, num_nbr=32, num_down=2, debug=False, print_time=False, device="cuda",
                 multilevel_neigh=False, threshold=256) -> None:
        if device != "cuda" and not str(device).startswith("cuda"):
            raise FknnError("FlashKNN-B200 runs on CUDA devices only")
        if not 1 <= int(num_nbr) <= 64:
            raise ValueError("num_nbr must lie in [1, 64]")
        if not 0 <= int(num_down) <= 8:
            raise ValueError("num_down must lie in [0, 8]")
        self.num_nbr = int(num_nbr)
        self.num_down = int(num_down)
        self.debug = debug
        self.print_time = print_time
        self.threshold = threshold
        self.multilevel_neigh = multilevel_neigh
        self.config = None  # optional fknn_config tuple; None = autotuned/default shape
        if self.debug:
            self.time_list = []

    # -------------------------------------------------------------- helpers
    @staticmethod
    def _check_modes(memory_mode, sorting_mode, candidate_mode, enable_skip, thread_group_size):
        if candidate_mode not in {"register", "shared"}:
            raise ValueError(
                f"candidate_mode must be 'register' or 'shared', got {candidate_mode!r}")
        if thread_group_size not in {None, 8, 16, 32}:
            raise ValueError(
                f"thread_group_size must be None, 8, 16, or 32, got {thread_group_size!r}")
        if (candidate_mode != "register" or not enable_skip) and not (
                memory_mode == "SM" and sorting_mode == "PS"):
            raise ValueError("candidate placement/skip ablations require memory_mode='SM' "
                             "and sorting_mode='PS'")
        if thread_group_size is not None and not (
                memory_mode == "SM" and sorting_mode == "PS" and candidate_mode == "register"
                and enable_skip):
            raise ValueError("fixed thread-group ablations require memory_mode='SM', "
                             "sorting_mode='PS', register candidates, and skip enabled")
        if memory_mode not in {"SM", "GM"}:
            raise ValueError(f"memory_mode must be 'SM' or 'GM', got {memory_mode!r}")
        if sorting_mode not in {"PS", "SS"}:
            raise ValueError(f"sorting_mode must be 'PS' or 'SS', got {sorting_mode!r}")

    def _record(self, kind, t0, extra=None):
        if not self.debug:
            return
        torch.cuda.synchronize()
        elapsed = time.perf_counter() - t0
        entry = {"total_s": elapsed, "query_type": kind}
        if extra:
            entry.update(extra)
        self.time_list.append(entry)
        if self.print_time:
            print(f"{kind}: {elapsed * 1e3:.3f} ms")

    # -------------------------------------------------------------- queries
    @torch.no_grad()
    def query(self, grid_coord, batch_idx, xyz=None, dynamic_load=True, cut_radius=math.inf,
              batch_for_prune=1, memory_mode="SM", sorting_mode="PS", candidate_mode="register",
              enable_skip=True, thread_group_size=None, traverse_info=None,
              return_distances=False, validate=False, graph=False):
        """Self query: the K nearest neighbours of every point among the points
        of the 27 parent cells around its own parent cell (parent = grid >>
        num_down).  Returns int64 [N, K] original indices; with
        ``return_distances`` returns (int32 indices, f32 squared distances).
        ``batch_for_prune`` and ``dynamic_load`` are accepted and unused, as in
        the reference kernel.  ``traverse_info[0]`` receives the mean number
        of candidates per parent cell (the points of its 27 neighbour cells),
        as FlashKnnWrapper.py:351-352 writes it: summed exactly on the device
        and rounded to FP32 (the reference takes an FP32 mean).  ``graph=True``
        replays a CUDA graph cached per input tensors (for small, repeated
        problems whose time is mostly kernel launches); the result then is
        the graph's own tensor, overwritten by the next such call.
        """
        self._check_modes(memory_mode, sorting_mode, candidate_mode, enable_skip,
                          thread_group_size)
        t0 = time.perf_counter() if self.debug else 0.0
        coords = xyz if xyz is not None else grid_coord.float()
        stats = [] if traverse_info is not None else None
        idx, dist = ops.knn_grid(
            coords, grid_coord, batch_idx, self.num_nbr, self.num_down,
            cut_r2=float(cut_radius) * float(cut_radius),
            idx_dtype=torch.int32 if return_distances else torch.int64,
            config=self.config, validate=validate, candidate_stats=stats, graph=graph)
        if traverse_info is not None:
            total, cells = stats[0]
            mean = total / cells if cells else float("nan")
            traverse_info[0] = float(np.float32(mean))
        self._record("query", t0, {"memory_mode": memory_mode, "sorting_mode": sorting_mode})
        return (idx, dist) if return_distances else idx

    @torch.no_grad()
    def selected_query(self, xyz, grid_coord, query_indices, batch_idx, dynamic_load=True,
                       cut_radius=math.inf, batch_for_prune=1, memory_mode="SM",
                       return_distances=False, validate=False):
        """Subset query (FlashKnnWrapper.py:646-849): rows follow
        ``query_indices``; candidates come from the full cloud; a row with
        fewer than K candidates is padded with the query's own index."""
        if memory_mode not in {"SM", "GM"}:
            raise ValueError(f"memory_mode must be 'SM' or 'GM', got {memory_mode!r}")
        t0 = time.perf_counter() if self.debug else 0.0
        coords = xyz if xyz is not None else grid_coord.float()
        idx, dist = ops.knn_grid(
            coords, grid_coord, batch_idx, self.num_nbr, self.num_down,
            cut_r2=float(cut_radius) * float(cut_radius), query_indices=query_indices,
            idx_dtype=torch.int32 if return_distances else torch.int64,
            config=self.config, validate=validate)
        self._record("selected_query", t0, {"memory_mode": memory_mode})
        return (idx, dist) if return_distances else idx

    @torch.no_grad()
    def back_query(self, xyz, sel_indices, query_grid_size, down_grid_size, batch_idx,
                   dynamic_load=True, memory_mode="SM"):
        """Dense-to-subset map (FlashKnnWrapper.py:459-644): for every point of
        ``xyz`` its ``num_nbr`` nearest points of the subset ``sel_indices``
        among the subset points in the 27 cells around its cell, cells =
        trunc(xyz / query_grid_size).  Returns positions in ``sel_indices``:
        K == 1: int64 [N] (memory_mode "SM") or [N, 1] ("GM"); K > 1:
        (int64 [N, K], f32 squared distances [N, K]), rows ascending (the
        reference leaves them in heap order).  Like the reference, raises
        AssertionError when some point has no subset point around it.
        ``down_grid_size`` and ``dynamic_load`` are accepted and unused, as
        in the reference."""
        del down_grid_size, dynamic_load
        if memory_mode not in {"SM", "GM"}:
            raise ValueError(f"memory_mode must be 'SM' or 'GM', got {memory_mode!r}")
        t0 = time.perf_counter() if self.debug else 0.0
        idx, dist, empty = ops.back_query(xyz.float(), sel_indices, query_grid_size,
                                          self.num_nbr, batch_idx, config=self.config,
                                          validate=True)
        if empty:
            raise AssertionError("some query points have no support point in their "
                                 "neighbourhood; consider a larger query_grid_size")
        self._record("back_query", t0, {"memory_mode": memory_mode})
        if self.num_nbr == 1:
            return idx.flatten() if memory_mode == "SM" else idx
        return idx, dist

    def rng_grid(self, rng, device="cuda"):
        """The 27 offsets (0,-1,+1)^3 in the reference's ij order, centre first."""
        if isinstance(rng, list):
            rng = torch.tensor(rng, dtype=torch.long, device=device)
        grid = torch.meshgrid(rng, rng, rng, indexing="ij")
        return torch.stack(grid, dim=-1).view(-1, 3)
