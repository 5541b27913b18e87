"""ctypes loader of the reference's nanoflann CPU kNN (TEST / BASELINE ONLY).

Built by oracle/build_ref.py (``build_nanoflann``) from the reference's
nanoflann.hpp into oracle/_ref/libref_nanoflann.so; see oracle/ref_nanoflann.cpp.
Exact FP32 kNN over each cloud of an offset batch; indices are local to the
cloud, rows unordered unless ``ordered`` (the reference's default,
Query/ThirdParty/nanoflannkdtree/TorchFlann/__init__.py:29,53-58).
"""
from __future__ import annotations

import ctypes
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(HERE, "_ref", "libref_nanoflann.so")
LEAF = 20  # the reference's max_leaf_size (TorchFlann/__init__.py:16)
_lib = None


def available() -> bool:
    return os.path.isfile(PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError("oracle/_ref/libref_nanoflann.so missing: run "
                                    "`python oracle/build_ref.py`")
        L = ctypes.CDLL(PATH)
        P, I32 = ctypes.c_void_p, ctypes.c_int
        L.rnf_build.restype = P
        L.rnf_build.argtypes = [P, P, I32, I32, I32]
        L.rnf_free.restype = None
        L.rnf_free.argtypes = [P]
        L.rnf_knn.restype = None
        L.rnf_knn.argtypes = [P, P, P, I32, I32, P, P, I32, I32]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def knn(xyz, offsets, k, q=None, q_offsets=None, ordered=False, nthreads=1):
    """Returns (idx uint32 [m, k] local to each cloud, dist f32 [m, k],
    build_seconds, query_seconds)."""
    L = lib()
    xyz = np.ascontiguousarray(xyz, np.float32)
    offsets = np.ascontiguousarray(offsets, np.int64)
    q = xyz if q is None else np.ascontiguousarray(q, np.float32)
    q_offsets = offsets if q_offsets is None else np.ascontiguousarray(q_offsets, np.int64)
    m = len(q)
    idx = np.empty((m, k), np.uint32)
    dist = np.empty((m, k), np.float32)
    t0 = time.perf_counter()
    h = L.rnf_build(_p(xyz), _p(offsets), len(offsets), LEAF, nthreads)
    t1 = time.perf_counter()
    try:
        L.rnf_knn(h, _p(q), _p(q_offsets), len(offsets), k, _p(idx), _p(dist),
                  1 if ordered else 0, nthreads)
        t2 = time.perf_counter()
    finally:
        L.rnf_free(h)
    return idx, dist, t1 - t0, t2 - t1
