"""ctypes binding of the CPU oracle (``gridknn_oracle.c``) -- TEST INFRASTRUCTURE.

Only the test suite, the smoke check and the benchmark's CPU-baseline leg use
this module.  The product library never imports it: the CUDA path has no CPU
fallback.  Every function here restates the reference algorithm cited in
``gridknn_oracle.c`` and works on numpy arrays.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborc.so")

_lib = None


def build() -> str:
    """Compile liborc.so with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or (
            os.path.getmtime(LIB_PATH)
            < os.path.getmtime(os.path.join(HERE, "gridknn_oracle.c"))
        ):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


P = ctypes.c_void_p
I64 = ctypes.c_int64
I32 = ctypes.c_int
F32 = ctypes.c_float


def _declare(L):
    L.orc_morton_key.restype = I64
    L.orc_morton_key.argtypes = [I64, I64, I64, I64]
    L.orc_morton_encode.restype = None
    L.orc_morton_encode.argtypes = [P, P, I64, P]
    L.orc_neighbor_keys.restype = None
    L.orc_neighbor_keys.argtypes = [P, P, I64, P]
    L.orc_argsort_i64.restype = None
    L.orc_argsort_i64.argtypes = [P, I64, P]
    L.orc_build_tables.restype = I64
    L.orc_build_tables.argtypes = [P, P, I64, I32, P, P, P, P, P, P]
    L.orc_query_tables.restype = I32
    L.orc_query_tables.argtypes = [P, P, P, P, I64, I32, F32, I32, P, P, P, I32]
    L.orc_selected_query_tables.restype = I32
    L.orc_selected_query_tables.argtypes = [P, P, P, P, P, P, I64, I32, F32, I32, P, P, P, I32]
    L.orc_knn_general.restype = I32
    L.orc_knn_general.argtypes = [P, P, P, I64, P, P, P, I64, I32, I32, F32, I32, P, P, P, I32]
    L.orc_knn_offsets.restype = I32
    L.orc_knn_offsets.argtypes = [P, P, I64, P, P, F32, I32, I32, F32, I32, P, P, I32]
    L.orc_brute_knn_f64.restype = I32
    L.orc_brute_knn_f64.argtypes = [P, P, I64, P, P, I32, P, P, I32]
    L.orc_backward_f64.restype = None
    L.orc_backward_f64.argtypes = [P, I64, P, I64, P, P, P, I32, P, P]
    L.orc_back_query_tables.restype = I32
    L.orc_back_query_tables.argtypes = [P, P, P, P, P, I64, I32, I32, P, P, I32]
    L.orc_back_query.restype = I32
    L.orc_back_query.argtypes = [P, I64, P, I64, P, F32, I32, I32, P, P, P, I32]
    L.orc_voxel_first.restype = I64
    L.orc_voxel_first.argtypes = [P, I64, P, F32, P]
    L.orc_adaptive_query.restype = I32
    L.orc_adaptive_query.argtypes = [P, P, I64, P, I32, I32, I32, I32, F32, I32, P, P, P, I32]


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


# Distance evaluation orders the oracle can reproduce (see gridknn_oracle.c).
VARIANT_FMA_YX = 0   # fma(dz,dz, fma(dy,dy, dx*dx))
VARIANT_FMA_XY = 1   # fma(dz,dz, fma(dx,dx, dy*dy))
VARIANT_ROUNDED = 2  # ((dx*dx + dy*dy) + dz*dz), no fused operations
# The order the CUDA kernels implement; the GPU parity tests check that the
# reference kernel's distances agree with it bit for bit.
DEFAULT_VARIANT = VARIANT_FMA_XY


def morton_key(x, y, z, b=0) -> int:
    return int(lib().orc_morton_key(int(x), int(y), int(z), int(b)))


def morton_encode(grid, batch=None):
    grid = _c(grid, np.int64)
    batch = _c(batch, np.int64)
    n = grid.shape[0]
    out = np.empty(n, np.int64)
    lib().orc_morton_encode(_ptr(grid), _ptr(batch), n, _ptr(out))
    return out


def neighbor_keys(grid_down, parent_batch=None):
    grid_down = _c(grid_down, np.int64)
    parent_batch = _c(parent_batch, np.int64)
    p = grid_down.shape[0]
    out = np.empty(p * 27, np.int64)
    lib().orc_neighbor_keys(_ptr(grid_down), _ptr(parent_batch), p, _ptr(out))
    return out


def build_tables(grid, batch, num_down):
    """Reference tables: dict(order, steps, neigh, cnt, grid_down, parent_batch)."""
    grid = _c(grid, np.int64)
    batch = _c(batch, np.int64)
    n = grid.shape[0]
    order = np.empty(n, np.int64)
    steps = np.empty(n + 1, np.int32)
    neigh = np.empty(max(n, 1) * 27, np.int32)
    cnt = np.empty(max(n, 1) * 28, np.int32)
    gd = np.empty(max(n, 1) * 3, np.int64)
    pb = np.empty(max(n, 1), np.int64)
    p = lib().orc_build_tables(_ptr(grid), _ptr(batch), n, num_down, _ptr(order),
                               _ptr(steps), _ptr(neigh), _ptr(cnt), _ptr(gd), _ptr(pb))
    return dict(order=order, steps=steps[: p + 1].copy(),
                neigh=neigh[: p * 27].reshape(p, 27).copy(),
                cnt=cnt[: p * 28].reshape(p, 28).copy(),
                grid_down=gd[: p * 3].reshape(p, 3).copy(), parent_batch=pb[:p].copy())


def query_tables(xyz_sorted, steps, neigh, cnt, k, cut_r2=np.inf,
                 variant=DEFAULT_VARIANT, idx_map=None, nthreads=0):
    """FlashKNN_Query_Dynamic_Load semantics: (idx int64 [n,K], dist f32 [n,K])."""
    xyz_sorted = _c(xyz_sorted, np.float32)
    steps = _c(steps, np.int32)
    neigh = _c(neigh, np.int32)
    cnt = _c(cnt, np.int32)
    idx_map = _c(idx_map, np.int64)
    n = xyz_sorted.shape[0]
    p = neigh.shape[0]
    idx = np.empty((n, k), np.int64)
    dist = np.empty((n, k), np.float32)
    rc = lib().orc_query_tables(_ptr(xyz_sorted), _ptr(steps), _ptr(neigh), _ptr(cnt), p,
                                k, float(cut_r2), variant, _ptr(idx_map), _ptr(idx),
                                _ptr(dist), nthreads)
    if rc != 0:
        raise ValueError(f"orc_query_tables failed with {rc}")
    return idx, dist


def selected_query_tables(xyz_sorted, qindex, steps, steps_query, neigh, cnt, k,
                          cut_r2=np.inf, variant=DEFAULT_VARIANT, idx_map=None,
                          nthreads=0):
    """FlashKNN_Selected_Query_DL semantics: rows follow qindex."""
    xyz_sorted = _c(xyz_sorted, np.float32)
    qindex = _c(qindex, np.int32)
    steps = _c(steps, np.int32)
    steps_query = _c(steps_query, np.int32)
    neigh = _c(neigh, np.int32)
    cnt = _c(cnt, np.int32)
    idx_map = _c(idx_map, np.int64)
    m = qindex.shape[0]
    p = neigh.shape[0]
    idx = np.empty((m, k), np.int64)
    dist = np.empty((m, k), np.float32)
    rc = lib().orc_selected_query_tables(_ptr(xyz_sorted), _ptr(qindex), _ptr(steps),
                                         _ptr(steps_query), _ptr(neigh), _ptr(cnt), p, k,
                                         float(cut_r2), variant, _ptr(idx_map), _ptr(idx),
                                         _ptr(dist), nthreads)
    if rc != 0:
        raise ValueError(f"orc_selected_query_tables failed with {rc}")
    return idx, dist


def knn_general(sxyz, sgrid, sbatch, qxyz, qgrid, qbatch, num_down, k,
                cut_r2=np.inf, pad=None, variant=DEFAULT_VARIANT, nthreads=0):
    """Original-index grid kNN for arbitrary queries; pad None means -1."""
    sxyz = _c(sxyz, np.float32)
    sgrid = _c(sgrid, np.int64)
    sbatch = _c(sbatch, np.int64)
    qxyz = _c(qxyz, np.float32)
    qgrid = _c(qgrid, np.int64)
    qbatch = _c(qbatch, np.int64)
    pad = _c(pad, np.int64)
    n, m = sxyz.shape[0], qxyz.shape[0]
    idx = np.empty((m, k), np.int32)
    dist = np.empty((m, k), np.float32)
    rc = lib().orc_knn_general(_ptr(sxyz), _ptr(sgrid), _ptr(sbatch), n, _ptr(qxyz),
                               _ptr(qgrid), _ptr(qbatch), m, num_down, k, float(cut_r2),
                               variant, _ptr(pad), _ptr(idx), _ptr(dist), nthreads)
    if rc != 0:
        raise ValueError(f"orc_knn_general failed with {rc}")
    return idx, dist


def knn_offsets(xyz, offsets, k, voxel, num_down=2, new_xyz=None, new_offsets=None,
                cut_r2=np.inf, variant=DEFAULT_VARIANT, nthreads=0):
    """Pointcept-style batched grid kNN (self query pads with own index)."""
    xyz = _c(xyz, np.float32)
    offsets = _c(offsets, np.int64)
    new_xyz = _c(new_xyz, np.float32)
    new_offsets = _c(new_offsets, np.int64)
    b = offsets.shape[0]
    m = (new_offsets[-1] if new_xyz is not None else offsets[-1]) if b else 0
    idx = np.empty((int(m), k), np.int32)
    dist = np.empty((int(m), k), np.float32)
    rc = lib().orc_knn_offsets(_ptr(xyz), _ptr(offsets), b, _ptr(new_xyz), _ptr(new_offsets),
                               float(voxel), num_down, k, float(cut_r2), variant, _ptr(idx),
                               _ptr(dist), nthreads)
    if rc != 0:
        raise ValueError(f"orc_knn_offsets failed with {rc}")
    return idx, dist


def brute_knn_f64(xyz, offsets, k, new_xyz=None, new_offsets=None, nthreads=0):
    """Exact FP64 kNN within each cloud: (idx int32, dist float64)."""
    xyz = _c(xyz, np.float32)
    offsets = _c(offsets, np.int64)
    new_xyz = _c(new_xyz, np.float32)
    new_offsets = _c(new_offsets, np.int64)
    b = offsets.shape[0]
    m = (new_offsets[-1] if new_xyz is not None else offsets[-1]) if b else 0
    idx = np.empty((int(m), k), np.int32)
    dist = np.empty((int(m), k), np.float64)
    rc = lib().orc_brute_knn_f64(_ptr(xyz), _ptr(offsets), b, _ptr(new_xyz),
                                 _ptr(new_offsets), k, _ptr(idx), _ptr(dist), nthreads)
    if rc != 0:
        raise ValueError(f"orc_brute_knn_f64 failed with {rc}")
    return idx, dist


def backward_f64(qxyz, pxyz, idx, dist, g):
    """FP64 analytic gradient of sum(g * d) with fixed indices."""
    qxyz = _c(qxyz, np.float32)
    pxyz = _c(pxyz, np.float32)
    idx = _c(idx, np.int32)
    dist = _c(dist, np.float32)
    g = _c(g, np.float64)
    m, k = idx.shape
    n = pxyz.shape[0]
    gq = np.empty((m, 3), np.float64)
    gp = np.empty((n, 3), np.float64)
    lib().orc_backward_f64(_ptr(qxyz), m, _ptr(pxyz), n, _ptr(idx), _ptr(dist), _ptr(g), k,
                           _ptr(gq), _ptr(gp))
    return gq, gp


def set_recall(pred, exact):
    """Row-wise set recall, repeated predictions counted once
    (Query/benchmark_s3dis.py:205-221)."""
    pred = np.sort(np.asarray(pred, np.int64), axis=1)
    exact = np.asarray(exact, np.int64)
    k = exact.shape[1]
    hits = np.zeros(exact.shape[0], np.float64)
    for r in range(exact.shape[0]):
        hits[r] = np.isin(exact[r], pred[r]).sum() / k
    return hits


def adaptive_query(grid, batch, k, xyz=None, min_factor=2, max_factor=8, max_shift=-1,
                   cut_r2=np.inf, variant=DEFAULT_VARIANT, nthreads=0):
    """Adaptive-neighbourhood self query (AdaptiveNeighborhoodFlashKNN):
    (levels int32 [n], idx int64 [n,K], dist f32 [n,K]) in input order."""
    grid = _c(grid, np.int64)
    batch = _c(batch, np.int64)
    xyz = _c(xyz, np.float32)
    n = grid.shape[0]
    levels = np.empty(n, np.int32)
    idx = np.empty((n, k), np.int64)
    dist = np.empty((n, k), np.float32)
    rc = lib().orc_adaptive_query(_ptr(grid), _ptr(batch), n, _ptr(xyz), k, min_factor,
                                  max_factor, max_shift, float(cut_r2), variant, _ptr(levels),
                                  _ptr(idx), _ptr(dist), nthreads)
    if rc != 0:
        raise ValueError(f"orc_adaptive_query failed with {rc}")
    return levels, idx, dist


def back_query_tables(xyz_h, xyz_l, steps_h, steps_l, neigh, k, variant=DEFAULT_VARIANT,
                      nthreads=0):
    """FlashKNN_Back_Query_DL semantics over the wrapper's tables: rows follow
    xyz_h, indices are rows of xyz_l; (idx int64 [nh,k], dist f32 [nh,k])."""
    xyz_h = _c(xyz_h, np.float32)
    xyz_l = _c(xyz_l, np.float32)
    steps_h = _c(steps_h, np.int32)
    steps_l = _c(steps_l, np.int32)
    neigh = _c(neigh, np.int32)
    p = neigh.shape[0]
    nh = xyz_h.shape[0]
    idx = np.empty((nh, k), np.int64)
    dist = np.empty((nh, k), np.float32)
    rc = lib().orc_back_query_tables(_ptr(xyz_h), _ptr(xyz_l), _ptr(steps_h), _ptr(steps_l),
                                     _ptr(neigh), p, k, variant, _ptr(idx), _ptr(dist), nthreads)
    if rc != 0:
        raise ValueError(f"orc_back_query_tables failed with {rc}")
    return idx, dist


def back_query(xyz, sel_indices, query_grid_size, k, batch=None, variant=DEFAULT_VARIANT,
               nthreads=0):
    """FlashKNN.back_query end to end: (idx int64 [n,k] positions in
    sel_indices, dist f32 [n,k], empty bool [n])."""
    xyz = _c(xyz, np.float32)
    sel_indices = _c(sel_indices, np.int64)
    batch = _c(batch, np.int64)
    n, m = xyz.shape[0], sel_indices.shape[0]
    idx = np.empty((n, k), np.int64)
    dist = np.empty((n, k), np.float32)
    empty = np.empty(n, np.int32)
    rc = lib().orc_back_query(_ptr(xyz), n, _ptr(sel_indices), m, _ptr(batch),
                              float(np.float32(query_grid_size)), k, variant, _ptr(idx),
                              _ptr(dist), _ptr(empty), nthreads)
    if rc != 0:
        raise ValueError(f"orc_back_query failed with {rc}")
    return idx, dist, empty.astype(bool)


def voxel_first(xyz, size, batch=None):
    """Voxel-first subsampling (one lowest-index point per occupied voxel):
    int64 indices, ascending."""
    xyz = _c(xyz, np.float32)
    batch = _c(batch, np.int64)
    n = xyz.shape[0]
    out = np.empty(max(n, 1), np.int64)
    c = lib().orc_voxel_first(_ptr(xyz), n, _ptr(batch), float(np.float32(size)), _ptr(out))
    return out[:c].copy()
