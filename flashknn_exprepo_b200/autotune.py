"""Autotuner of the query kernel's launch shape.

The top-K kernel has four shape knobs (``fknn_config``): warps per CTA
(queries per CTA, 32 per warp), the candidate tile staged in shared memory
per warp (``tile_records``; groups with more candidates stream tile by
tile), how many lanes may share one query when a group is larger than a
tile (``min_candidates_per_lane``), and the shared-memory staging depth (1:
a warp stages a work item's candidates and then scans them; 2: two tiles
per warp, the next item's bulk copies in flight during the scan, at twice
the tile memory, hence fewer resident warps).  The best shape depends on K (register
list length, hence occupancy) and on point density (candidates per query,
hence tile fill and the chunked path).  ``tune_offsets`` times a
coarse-to-fine grid of shapes on the caller's own workload with CUDA events
and keeps the fastest per (GPU, K bucket, density bucket): the density is
the mean number of points per occupied parent cell, in powers of two.  The
cache lives in memory and, when ``FKNN_TUNE_CACHE`` names a file, in JSON.
"""
from __future__ import annotations

import json
import math
import os
import threading

import torch

from . import _lib, ops

WARPS = (2, 4, 8)
TILES = (256, 384, 448, 512, 640, 768, 1024)
LANE_SHARES = (4, 8, 16)
DEPTHS = (1, 2)
DEFAULT = (4, 448, 8, 0, 1)

_cache: dict = {}
_lock = threading.Lock()


def k_bucket(k: int) -> int:
    """Register-list length the kernel uses for K (1, 2, 4, ..., 64)."""
    b = 1
    while b < k:
        b <<= 1
    return b


def density_bucket(xyz: torch.Tensor, offset: torch.Tensor, voxel: float, num_down: int) -> int:
    """log2 of the mean points per occupied parent cell (rounded), from the
    same voxelisation as the query (floor(x * (1/voxel)) >> num_down), clouds
    kept apart.  One synchronisation."""
    inv = torch.tensor(1.0, dtype=torch.float32) / torch.tensor(voxel, dtype=torch.float32)
    g = torch.floor(xyz * inv.to(xyz.device)).long() >> num_down
    cloud = torch.bucketize(torch.arange(len(xyz), device=xyz.device), offset, right=True)
    g = g - g.min(0).values
    span = g.max(0).values + 1
    key = ((cloud * span[0] + g[:, 0]) * span[1] + g[:, 1]) * span[2] + g[:, 2]
    cells = int(torch.unique(key).numel())
    return int(round(math.log2(max(len(xyz), 1) / max(cells, 1))))


def _key(dev: torch.device, k: int, density: int) -> str:
    return f"{torch.cuda.get_device_name(dev)}|k{k_bucket(k)}|d{density}"


def _load_file():
    path = os.environ.get("FKNN_TUNE_CACHE")
    if path and os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def _save_file():
    path = os.environ.get("FKNN_TUNE_CACHE")
    if path:
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(_cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)


def lookup(dev: torch.device, k: int, density: int):
    """Cached shape for (GPU, K bucket, density bucket), or None."""
    with _lock:
        if not _cache:
            _cache.update(_load_file())
        hit = _cache.get(_key(dev, k, density))
    return _lib.FknnConfig(*hit["config"]) if hit else None


def _time(fn, reps: int) -> float:
    fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def tune_offsets(xyz, offset, k, voxel, num_down=2, reps=3, force=False):
    """Fastest launch shape for this self-query workload (and its class).

    Times every (warps, tile, depth) triple with 8 lanes per query share,
    then the lane shares for the best triple; returns the FknnConfig and
    records it for (GPU, K bucket, density bucket).  Results are identical for every shape
    (the shape changes the schedule, never the answer)."""
    dev = xyz.device
    density = density_bucket(xyz, offset, voxel, num_down)
    if not force:
        hit = lookup(dev, k, density)
        if hit is not None:
            return hit
    times = {}

    def run(cfg):
        """ms per call, or None for a shape the library rejects (shared
        memory beyond a CTA's)."""
        try:
            return _time(lambda: ops.knn_offsets(xyz, offset, k, voxel, num_down,
                                                 config=_lib.FknnConfig(*cfg)), reps)
        except _lib.FknnError:
            return None

    for w in WARPS:
        for t in TILES:
            for depth in DEPTHS:
                ms = run((w, t, 8, 0, depth))
                if ms is not None:
                    times[(w, t, 8, 0, depth)] = ms
    best = min(times, key=times.get)
    for share in LANE_SHARES:
        cfg = (best[0], best[1], share, 0, best[4])
        if cfg not in times:
            ms = run(cfg)
            if ms is not None:
                times[cfg] = ms
    best = min(times, key=times.get)
    with _lock:
        _cache[_key(dev, k, density)] = {"config": list(best), "ms": times[best],
                                         "default_ms": times.get(DEFAULT)}
        _save_file()
    return _lib.FknnConfig(*best)


def last_results() -> dict:
    """The in-memory cache: key -> {config, ms, default_ms}."""
    with _lock:
        return dict(_cache)
