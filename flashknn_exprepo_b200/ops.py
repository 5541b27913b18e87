"""Tensor-level entry points over the C ABI (one call = one stream of launches).

Every function takes CUDA tensors, launches on the current stream, and
returns new tensors.  Nothing here synchronises unless ``validate=True``,
which reads the device status word once and raises on any device-side
problem (coordinates outside the Morton range, bad tables, ...).
"""
from __future__ import annotations

import collections
import ctypes
import math
import threading

import torch

from . import _lib
from ._lib import FknnError, check, ptr, stream_handle


def _require(t: torch.Tensor, name: str, dtype, ndim=None, cols=None) -> torch.Tensor:
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if not t.is_cuda:
        raise FknnError(f"{name} must be a CUDA tensor (FlashKNN-B200 has no CPU path)")
    if t.dtype != dtype:
        t = t.to(dtype)
    if ndim is not None and t.dim() != ndim:
        raise ValueError(f"{name} must have {ndim} dimensions, got shape {tuple(t.shape)}")
    if cols is not None and t.shape[-1] != cols:
        raise ValueError(f"{name} must have shape [N, {cols}], got {tuple(t.shape)}")
    return t.contiguous()


def _config_ptr(config):
    if config is None:
        return None, None
    if isinstance(config, _lib.FknnConfig):
        c = config
    else:
        c = _lib.FknnConfig(*config)
    return c, ctypes.byref(c)


class _GraphCache:
    """Captured pipelines for ``graph=True`` calls, per host thread (LRU).

    A small problem spends most of its time launching its dozen kernels;
    replaying them from one CUDA graph removes the host-side launch cost.
    An entry is keyed by everything the launches depend on -- the entry
    point, the device, the input pointers and sizes, K, the grid parameters
    and the launch shape -- and owns its workspace and output tensors: the
    tensors a graph call returns are overwritten by the next call with the
    same key (clone them to keep them).  Data-dependent sizes (cells, work
    items) stay on the device, so one capture serves any point values."""

    def __init__(self, capacity=16):
        self._local = threading.local()
        self.capacity = capacity

    def _entries(self):
        e = getattr(self._local, "entries", None)
        if e is None:
            e = self._local.entries = collections.OrderedDict()
        return e

    def run(self, key, dev, ws_bytes, make_outputs, launch):
        entries = self._entries()
        hit = entries.get(key)
        if hit is None:
            ws = torch.empty(max(int(ws_bytes), 256), dtype=torch.uint8, device=dev)
            cur = torch.cuda.current_stream(dev)
            side = torch.cuda.Stream(dev)
            side.wait_stream(cur)
            with torch.cuda.stream(side):
                launch(ws, *make_outputs())  # loads the kernels, fills the launch cache
                graph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(graph, stream=side):
                    outs = make_outputs()
                    launch(ws, *outs)
            cur.wait_stream(side)
            hit = (graph, outs, ws)
            entries[key] = hit
            while len(entries) > self.capacity:
                entries.popitem(last=False)
        else:
            entries.move_to_end(key)
        hit[0].replay()
        return hit[1], hit[2]

    def clear(self):
        self._entries().clear()


GRAPHS = _GraphCache()


def knn_offsets(xyz, offset, k, voxel, num_down=2, new_xyz=None, new_offset=None,
                cut_r2=math.inf, config=None, validate=False, graph=False):
    """Pointcept-style batched grid kNN.  Returns (idx int32 [m,k], dist2 f32 [m,k]).

    ``graph=True`` replays a cached CUDA graph of the whole pipeline (captured
    on the first call with these inputs); the returned tensors are the
    graph's own and are overwritten by the next such call."""
    return _offsets_call("fknn_knn_offsets", xyz, offset, k, voxel, num_down, new_xyz,
                         new_offset, float(cut_r2), config, validate, graph)


def ball_query_offsets(xyz, offset, nsample, max_radius, voxel, num_down=2, new_xyz=None,
                       new_offset=None, config=None, validate=False):
    """The nsample nearest points within max_radius among the 27 parent cells
    (fknn_ball_query).  Returns (idx int32 [m,nsample], dist2 f32), rows
    padded with (-1, +inf)."""
    return _offsets_call("fknn_ball_query", xyz, offset, nsample, voxel, num_down, new_xyz,
                         new_offset, float(max_radius), config, validate)


def _offsets_call(entry, xyz, offset, k, voxel, num_down, new_xyz, new_offset, last, config,
                  validate, graph=False):
    lib = _lib.load()
    xyz = _require(xyz, "xyz", torch.float32, 2, 3)
    dev = xyz.device
    offset = _require(offset, "offset", torch.int64, 1)
    general = new_xyz is not None
    if general:
        new_xyz = _require(new_xyz, "new_xyz", torch.float32, 2, 3)
        if new_offset is None:
            raise ValueError("new_offset is required with new_xyz")
        new_offset = _require(new_offset, "new_offset", torch.int64, 1)
        if new_offset.numel() != offset.numel():
            raise ValueError("offset and new_offset must describe the same number of clouds")
    n = xyz.shape[0]
    m = new_xyz.shape[0] if general else n
    b = offset.numel()
    kind = _lib.QUERY_GENERAL if general else _lib.QUERY_SELF
    nbytes = lib.fknn_workspace_bytes(n, m, max(b, 1), kind)
    c, cfg = _config_ptr(config)

    def outputs():
        return (torch.empty((m, k), dtype=torch.int32, device=dev),
                torch.empty((m, k), dtype=torch.float32, device=dev))

    def launch(ws, idx, dist):
        rc = getattr(lib, entry)(ptr(xyz), n, ptr(offset), b, ptr(new_xyz), m, ptr(new_offset),
                                 k, float(voxel), num_down, last, ptr(idx), ptr(dist), ptr(ws),
                                 ws.numel(), cfg, stream_handle(dev))
        check(rc, entry)

    if graph:
        key = (entry, dev.index, ptr(xyz), n, ptr(offset), b, ptr(new_xyz), m, ptr(new_offset),
               k, float(voxel), num_down, last, None if c is None else c.as_tuple())
        (idx, dist), ws = GRAPHS.run(key, dev, nbytes, outputs, launch)
    else:
        ws = _lib.WORKSPACE.get(nbytes, dev)
        idx, dist = outputs()
        launch(ws, idx, dist)
    if validate:
        _lib.raise_on_status(ws, entry)
    return idx, dist


def knn_grid(xyz, grid_coord, batch_idx, k, num_down=2, cut_r2=math.inf, query_indices=None,
             idx_dtype=torch.int64, config=None, validate=False, candidate_stats=None,
             graph=False):
    """FlashKNN.query / selected_query on caller-voxelised grid coordinates.

    Returns (idx [m,k] of ``idx_dtype`` in original point numbering, dist2 f32).
    With ``candidate_stats`` (a list) a self query appends (candidate total,
    parent cells) read back from the device (one synchronisation).
    ``graph=True`` replays a cached CUDA graph, as ``knn_offsets``.
    """
    lib = _lib.load()
    grid_coord = _require(grid_coord, "grid_coord", torch.int64, 2, 3)
    dev = grid_coord.device
    xyz = _require(xyz, "xyz", torch.float32, 2, 3)
    if batch_idx is not None:
        batch_idx = _require(batch_idx, "batch_idx", torch.int64, 1)
        if batch_idx.numel() != grid_coord.shape[0]:
            raise ValueError("batch_idx must have one entry per point")
    if xyz.shape[0] != grid_coord.shape[0]:
        raise ValueError("xyz and grid_coord must have the same number of points")
    n = grid_coord.shape[0]
    selected = query_indices is not None
    if selected:
        query_indices = _require(query_indices, "query_indices", torch.int64, 1)
    m = query_indices.numel() if selected else n
    if idx_dtype not in (torch.int32, torch.int64):
        raise ValueError("idx_dtype must be torch.int32 or torch.int64")
    kind = _lib.QUERY_SELECTED if selected else _lib.QUERY_SELF
    nbytes = lib.fknn_workspace_bytes(n, m, 32768, kind)
    c, cfg = _config_ptr(config)
    bits = 64 if idx_dtype == torch.int64 else 32

    def outputs():
        return (torch.empty((m, k), dtype=idx_dtype, device=dev),
                torch.empty((m, k), dtype=torch.float32, device=dev))

    def launch(ws, idx, dist):
        rc = lib.fknn_knn_grid(ptr(xyz), ptr(grid_coord), ptr(batch_idx), n, ptr(query_indices),
                               m, k, num_down, float(cut_r2), bits, ptr(idx), ptr(dist),
                               ptr(ws), ws.numel(), cfg, stream_handle(dev))
        check(rc, "fknn_knn_grid")

    if graph:
        key = ("fknn_knn_grid", dev.index, ptr(xyz), ptr(grid_coord), ptr(batch_idx), n,
               ptr(query_indices), m, k, num_down, float(cut_r2), bits,
               None if c is None else c.as_tuple())
        (idx, dist), ws = GRAPHS.run(key, dev, nbytes, outputs, launch)
    else:
        ws = _lib.WORKSPACE.get(nbytes, dev)
        idx, dist = outputs()
        launch(ws, idx, dist)
    if validate:
        _lib.raise_on_status(ws, "knn_grid")
    if candidate_stats is not None:
        candidate_stats.append(_lib.candidate_stats(ws))
    return idx, dist


def back_query(xyz, sel_indices, query_grid_size, k, batch_idx=None, idx_dtype=torch.int64,
               config=None, validate=False, status_into=None):
    """FlashKNN.back_query kernels: for every point of ``xyz`` the k nearest
    points of the subset ``sel_indices`` in the 27 cells around its cell
    (cells = trunc(xyz / query_grid_size)).  Returns (idx [n,k] positions in
    ``sel_indices``, dist2 f32 [n,k], empty) where ``empty`` is True when some
    point had no subset point around it (its row is (-1, +inf)).  With
    ``status_into`` (an int32 CUDA tensor of one element) the device status
    word is OR-ed into it on the stream instead of being read back, so
    several calls can be checked with one synchronisation."""
    lib = _lib.load()
    xyz = _require(xyz, "xyz", torch.float32, 2, 3)
    dev = xyz.device
    n = xyz.shape[0]
    sel_indices = _require(sel_indices, "sel_indices", torch.int64, 1)
    m = sel_indices.numel()
    if batch_idx is not None:
        batch_idx = _require(batch_idx, "batch_idx", torch.int64, 1)
        if batch_idx.numel() != n:
            raise ValueError("batch_idx must have one entry per point")
    if idx_dtype not in (torch.int32, torch.int64):
        raise ValueError("idx_dtype must be torch.int32 or torch.int64")
    idx = torch.empty((n, k), dtype=idx_dtype, device=dev)
    dist = torch.empty((n, k), dtype=torch.float32, device=dev)
    ws = _lib.WORKSPACE.get(lib.fknn_back_query_workspace_bytes(n, m), dev)
    _, cfg = _config_ptr(config)
    rc = lib.fknn_back_query(ptr(xyz), n, ptr(sel_indices), m, ptr(batch_idx),
                             float(query_grid_size), k, 64 if idx_dtype == torch.int64 else 32,
                             ptr(idx), ptr(dist), ptr(ws), ws.numel(), cfg, stream_handle(dev))
    check(rc, "fknn_back_query")
    if status_into is not None:
        status_into.bitwise_or_(ws[:4].view(torch.int32))
    empty = None
    if validate:
        _lib.raise_on_status(ws, "back_query")
        empty = bool(_lib.read_status(ws) & _lib.DEVICE_NO_CANDIDATES)
    return idx, dist, empty


def group_features(feat, idx, xyz=None, new_xyz=None, with_xyz=False, validate=False):
    """out [m,k,c(+3)]: rows of feat (and xyz[t] - new_xyz[i] first with
    with_xyz) gathered by idx; idx < 0 gives zeros (fknn_group_features)."""
    lib = _lib.load()
    feat = _require(feat, "feat", torch.float32, 2)
    dev = feat.device
    idx = _require(idx, "idx", torch.int32, 2)
    n, c = feat.shape
    m, k = idx.shape
    if with_xyz:
        xyz = _require(xyz, "xyz", torch.float32, 2, 3)
        new_xyz = _require(new_xyz, "new_xyz", torch.float32, 2, 3)
        if xyz.shape[0] != n or new_xyz.shape[0] != m:
            raise ValueError("xyz must have one row per feature row, new_xyz one per idx row")
    out = torch.empty((m, k, c + (3 if with_xyz else 0)), dtype=torch.float32, device=dev)
    ws = _lib.WORKSPACE.get(lib.fknn_group_workspace_bytes(m, k, n), dev)
    rc = lib.fknn_group_features(ptr(feat), n, c, ptr(idx), m, k,
                                 ptr(xyz) if with_xyz else None,
                                 ptr(new_xyz) if with_xyz else None, 1 if with_xyz else 0,
                                 ptr(out), ptr(ws), ws.numel(), stream_handle(dev))
    check(rc, "fknn_group_features")
    if validate:
        _lib.raise_on_status(ws, "group_features")
    return out


def group_backward(grad_out, idx, n, c, with_xyz=False, grad_feat=None, grad_xyz=None,
                   accumulate_xyz=False, grad_new_xyz=None, accumulate_new_xyz=False):
    """Deterministic gradients of group_features (fknn_group_backward)."""
    lib = _lib.load()
    grad_out = _require(grad_out, "grad_out", torch.float32, 3)
    dev = grad_out.device
    idx = _require(idx, "idx", torch.int32, 2)
    m, k = idx.shape
    ws = _lib.WORKSPACE.get(lib.fknn_group_workspace_bytes(m, k, n), dev)
    rc = lib.fknn_group_backward(ptr(grad_out), n, c, ptr(idx), m, k, 1 if with_xyz else 0,
                                 ptr(grad_feat), ptr(grad_xyz), 1 if accumulate_xyz else 0,
                                 ptr(grad_new_xyz), 1 if accumulate_new_xyz else 0, ptr(ws),
                                 ws.numel(), stream_handle(dev))
    check(rc, "fknn_group_backward")
    return grad_feat, grad_xyz, grad_new_xyz


def voxel_first(xyz, voxel, batch_idx=None, validate=False):
    """Voxel-first subsampling: the lowest index of every occupied voxel
    (voxel = floor(xyz * (1 / voxel))), ascending int64.  Reads the count back
    (one synchronisation)."""
    lib = _lib.load()
    xyz = _require(xyz, "xyz", torch.float32, 2, 3)
    dev = xyz.device
    n = xyz.shape[0]
    if batch_idx is not None:
        batch_idx = _require(batch_idx, "batch_idx", torch.int64, 1)
        if batch_idx.numel() != n:
            raise ValueError("batch_idx must have one entry per point")
    out = torch.empty(n, dtype=torch.int64, device=dev)
    count = torch.empty(1, dtype=torch.int64, device=dev)
    ws = _lib.WORKSPACE.get(lib.fknn_voxel_first_workspace_bytes(n), dev)
    rc = lib.fknn_voxel_first(ptr(xyz), n, ptr(batch_idx), float(voxel), ptr(out), ptr(count),
                              ptr(ws), ws.numel(), stream_handle(dev))
    check(rc, "fknn_voxel_first")
    # one read-back for both the count and the device status word
    status = ws[:4].view(torch.int32).to(torch.int64)
    got = torch.cat([count, status]).cpu()
    bits = int(got[1]) & ~_lib.DEVICE_NO_CANDIDATES
    if validate and bits:
        raise FknnError(f"voxel_first: device reported {_lib.status_text(bits)} (status {bits})")
    return out[: int(got[0])]


def adaptive_query(grid_coord, batch_idx, k, xyz=None, min_factor=2, max_factor=8,
                   max_shift=None, cut_r2=math.inf, idx_dtype=torch.int64, config=None,
                   want_levels=False, validate=False):
    """AdaptiveNeighborhoodFlashKNN.query: per-point octree level, exact top-K
    over the 27 same-level nodes.  Returns (idx [n,k] of ``idx_dtype`` in
    input numbering, dist2 f32 [n,k], levels int8 [n] or None)."""
    lib = _lib.load()
    grid_coord = _require(grid_coord, "grid_coord", torch.int64, 2, 3)
    dev = grid_coord.device
    n = grid_coord.shape[0]
    if batch_idx is not None:
        batch_idx = _require(batch_idx, "batch_idx", torch.int64, 1)
        if batch_idx.numel() != n:
            raise ValueError("batch_idx must have one entry per point")
    if xyz is not None:
        xyz = _require(xyz, "xyz", torch.float32, 2, 3)
        if xyz.shape[0] != n:
            raise ValueError("xyz and grid_coord must have the same number of points")
    if idx_dtype not in (torch.int32, torch.int64):
        raise ValueError("idx_dtype must be torch.int32 or torch.int64")
    idx = torch.empty((n, k), dtype=idx_dtype, device=dev)
    dist = torch.empty((n, k), dtype=torch.float32, device=dev)
    levels = torch.empty(n, dtype=torch.int8, device=dev) if want_levels else None
    ws = _lib.WORKSPACE.get(lib.fknn_adaptive_workspace_bytes(n), dev)
    _, cfg = _config_ptr(config)
    rc = lib.fknn_adaptive_query(ptr(grid_coord), ptr(batch_idx), n, ptr(xyz), k, int(min_factor),
                                 int(max_factor), -1 if max_shift is None else int(max_shift),
                                 float(cut_r2), 64 if idx_dtype == torch.int64 else 32, ptr(idx),
                                 ptr(dist), ptr(levels), ptr(ws), ws.numel(), cfg,
                                 stream_handle(dev))
    check(rc, "fknn_adaptive_query")
    if validate:
        _lib.raise_on_status(ws, "adaptive_query")
    return idx, dist, levels


def query_tables(xyz_sorted, steps, neigh, cnt, k, cut_r2=math.inf, config=None,
                 validate=False):
    """Reference table ABI (FlashKNN_Query_Dynamic_Load): sorted-space (idx, dist)."""
    lib = _lib.load()
    xyz_sorted = _require(xyz_sorted, "xyz_sorted", torch.float32, 2, 3)
    dev = xyz_sorted.device
    steps = _require(steps, "steps", torch.int32, 1)
    neigh = _require(neigh, "neigh", torch.int32, 2, 27)
    cnt = _require(cnt, "cnt", torch.int32, 2, 28)
    n, p = xyz_sorted.shape[0], neigh.shape[0]
    if steps.numel() != p + 1 or cnt.shape[0] != p:
        raise ValueError("steps must have P+1 entries and cnt P rows")
    idx = torch.empty((n, k), dtype=torch.int32, device=dev)
    dist = torch.empty((n, k), dtype=torch.float32, device=dev)
    ws = _lib.WORKSPACE.get(lib.fknn_tables_workspace_bytes(n, n, p), dev)
    _, cfg = _config_ptr(config)
    rc = lib.fknn_query_tables(ptr(xyz_sorted), n, ptr(steps), ptr(neigh), ptr(cnt), p, k,
                               float(cut_r2), ptr(idx), ptr(dist), ptr(ws), ws.numel(), cfg,
                               stream_handle(dev))
    check(rc, "fknn_query_tables")
    if validate:
        _lib.raise_on_status(ws, "query_tables")
    return idx, dist


def general_query_tables(xyz_support, xyz_query, steps, steps_query, neigh, cnt, k,
                         pad_index=None, cut_r2=math.inf, config=None, validate=False):
    """Separate query points over caller tables (FlashKNN_Query_GM and the
    back-query table kernels): (idx int32 [m,k] rows of xyz_support, dist2)."""
    lib = _lib.load()
    xyz_support = _require(xyz_support, "xyz_support", torch.float32, 2, 3)
    dev = xyz_support.device
    xyz_query = _require(xyz_query, "xyz_query", torch.float32, 2, 3)
    steps = _require(steps, "steps", torch.int32, 1)
    steps_query = _require(steps_query, "steps_query", torch.int32, 1)
    neigh = _require(neigh, "neigh", torch.int32, 2, 27)
    cnt = _require(cnt, "cnt", torch.int32, 2, 28)
    n, m, p = xyz_support.shape[0], xyz_query.shape[0], neigh.shape[0]
    if steps.numel() != p + 1 or steps_query.numel() != p + 1 or cnt.shape[0] != p:
        raise ValueError("steps and steps_query must have P+1 entries and cnt P rows")
    if pad_index is not None:
        pad_index = _require(pad_index, "pad_index", torch.int32, 1)
        if pad_index.numel() != m:
            raise ValueError("pad_index must have one entry per query")
    idx = torch.empty((m, k), dtype=torch.int32, device=dev)
    dist = torch.empty((m, k), dtype=torch.float32, device=dev)
    ws = _lib.WORKSPACE.get(lib.fknn_tables_workspace_bytes(n, m, p), dev)
    _, cfg = _config_ptr(config)
    rc = lib.fknn_general_query_tables(ptr(xyz_support), n, ptr(xyz_query), m, ptr(pad_index),
                                       ptr(steps), ptr(steps_query), ptr(neigh), ptr(cnt), p, k,
                                       float(cut_r2), ptr(idx), ptr(dist), ptr(ws), ws.numel(),
                                       cfg, stream_handle(dev))
    check(rc, "fknn_general_query_tables")
    if validate:
        _lib.raise_on_status(ws, "general_query_tables")
    return idx, dist


def selected_query_tables(xyz_sorted, qindex, steps, steps_query, neigh, cnt, k,
                          cut_r2=math.inf, config=None, validate=False):
    """Reference table ABI (FlashKNN_Selected_Query_DL): rows follow qindex."""
    lib = _lib.load()
    xyz_sorted = _require(xyz_sorted, "xyz_sorted", torch.float32, 2, 3)
    dev = xyz_sorted.device
    qindex = _require(qindex, "qindex", torch.int32, 1)
    steps = _require(steps, "steps", torch.int32, 1)
    steps_query = _require(steps_query, "steps_query", torch.int32, 1)
    neigh = _require(neigh, "neigh", torch.int32, 2, 27)
    cnt = _require(cnt, "cnt", torch.int32, 2, 28)
    n, m, p = xyz_sorted.shape[0], qindex.numel(), neigh.shape[0]
    idx = torch.empty((m, k), dtype=torch.int32, device=dev)
    dist = torch.empty((m, k), dtype=torch.float32, device=dev)
    ws = _lib.WORKSPACE.get(lib.fknn_tables_workspace_bytes(n, m, p), dev)
    _, cfg = _config_ptr(config)
    rc = lib.fknn_selected_query_tables(ptr(xyz_sorted), n, ptr(qindex), m, ptr(steps),
                                        ptr(steps_query), ptr(neigh), ptr(cnt), p, k,
                                        float(cut_r2), ptr(idx), ptr(dist), ptr(ws), ws.numel(),
                                        cfg, stream_handle(dev))
    check(rc, "fknn_selected_query_tables")
    if validate:
        _lib.raise_on_status(ws, "selected_query_tables")
    return idx, dist


def morton_encode(grid_coord, batch_idx=None):
    """FlashKNN_Morton_Encode: int64 keys of [N,3] grid coordinates."""
    lib = _lib.load()
    grid_coord = _require(grid_coord, "grid_coord", torch.int64, 2, 3)
    if batch_idx is not None:
        batch_idx = _require(batch_idx, "batch_idx", torch.int64, 1)
    keys = torch.empty(grid_coord.shape[0], dtype=torch.int64, device=grid_coord.device)
    check(lib.fknn_morton_encode(ptr(grid_coord), ptr(batch_idx), grid_coord.shape[0], ptr(keys),
                                 stream_handle(grid_coord.device)), "fknn_morton_encode")
    return keys


def morton_neighbor_keys(grid_coord_down, parent_batch=None):
    """FlashKNN_Morton_Neighbor_Keys: [P*27] keys, centre first."""
    lib = _lib.load()
    grid_coord_down = _require(grid_coord_down, "grid_coord_down", torch.int64, 2, 3)
    if parent_batch is not None:
        parent_batch = _require(parent_batch, "parent_batch", torch.int64, 1)
    p = grid_coord_down.shape[0]
    keys = torch.empty(p * 27, dtype=torch.int64, device=grid_coord_down.device)
    check(lib.fknn_morton_neighbor_keys(ptr(grid_coord_down), ptr(parent_batch), p, ptr(keys),
                                        stream_handle(grid_coord_down.device)),
          "fknn_morton_neighbor_keys")
    return keys


def build_tables(grid_coord, batch_idx, num_down):
    """The reference's table construction on the device.

    Returns dict(order int64 [N], steps int32 [P+1], neigh int32 [P,27],
    cnt int32 [P,28]).  Reads P back to the host (one synchronisation).
    """
    lib = _lib.load()
    grid_coord = _require(grid_coord, "grid_coord", torch.int64, 2, 3)
    dev = grid_coord.device
    if batch_idx is not None:
        batch_idx = _require(batch_idx, "batch_idx", torch.int64, 1)
    n = grid_coord.shape[0]
    order = torch.empty(n, dtype=torch.int64, device=dev)
    steps = torch.empty(n + 1, dtype=torch.int32, device=dev)
    neigh = torch.empty(max(n, 1) * 27, dtype=torch.int32, device=dev)
    cnt = torch.empty(max(n, 1) * 28, dtype=torch.int32, device=dev)
    n_parents = torch.zeros(1, dtype=torch.int64, device=dev)
    ws = _lib.WORKSPACE.get(lib.fknn_build_tables_workspace_bytes(n), dev)
    check(lib.fknn_build_tables(ptr(grid_coord), ptr(batch_idx), n, num_down, ptr(order),
                                ptr(steps), ptr(neigh), ptr(cnt), ptr(n_parents), ptr(ws),
                                ws.numel(), stream_handle(dev)), "fknn_build_tables")
    p = int(n_parents.item())
    return dict(order=order, steps=steps[: p + 1], neigh=neigh[: p * 27].view(p, 27),
                cnt=cnt[: p * 28].view(p, 28))


def backward(q_xyz, p_xyz, idx, dist, grad_dist, grad_q=None, grad_p=None, accumulate=False):
    """Gradients of sum(grad_dist * dist) w.r.t. the query and support coordinates.

    grad_q / grad_p: output tensors (allocated when None and requested through
    the ``want`` semantics of the caller).  Pass the same tensor for both with
    ``accumulate=True`` to get their sum (self query).
    """
    lib = _lib.load()
    q_xyz = _require(q_xyz, "q_xyz", torch.float32, 2, 3)
    p_xyz = _require(p_xyz, "p_xyz", torch.float32, 2, 3)
    dev = q_xyz.device
    idx = _require(idx, "idx", torch.int32, 2)
    dist = _require(dist, "dist", torch.float32, 2)
    grad_dist = _require(grad_dist, "grad_dist", torch.float32, 2)
    m, k = idx.shape
    n = p_xyz.shape[0]
    ws = _lib.WORKSPACE.get(lib.fknn_backward_workspace_bytes(m, n, k), dev)
    check(lib.fknn_backward(ptr(q_xyz), m, ptr(p_xyz), n, ptr(idx), ptr(dist), ptr(grad_dist), k,
                            ptr(grad_q), ptr(grad_p), 1 if accumulate else 0, ptr(ws),
                            ws.numel(), stream_handle(dev)), "fknn_backward")
    return grad_q, grad_p


def last_launch_count() -> int:
    """Kernels launched by the last successful C-ABI call on this process."""
    return int(_lib.load().fknn_last_launch_count())
