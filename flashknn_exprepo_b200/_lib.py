"""ctypes binding of libfknn.so, the C ABI declared in include/fknn.h.

There is no fallback: if the library or a CUDA device is missing, every
entry point raises :class:`FknnError`.
"""
from __future__ import annotations

import ctypes
import os
import threading

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfknn.so")

FKNN_OK = 0
FKNN_ERR_ARG = -1
FKNN_ERR_K = -2
FKNN_ERR_WORKSPACE = -3
FKNN_ERR_CUDA = -4
FKNN_ERR_SIZE = -5
FKNN_ERR_NUM_DOWN = -6
FKNN_ERR_SCRATCH_LIMIT = -7

DEVICE_COORD_RANGE = 1
DEVICE_BAD_TABLE = 2
DEVICE_TIMEOUT = 4
DEVICE_BATCH_RANGE = 8
DEVICE_NO_CANDIDATES = 16  # informational: general / back queries pad such rows
DEVICE_COPY_IN_FLIGHT = 32

QUERY_SELF = 0
QUERY_SELECTED = 1
QUERY_GENERAL = 2

_STATUS_TEXT = {
    DEVICE_COORD_RANGE: "a grid coordinate lies outside [-2^15, 2^15)",
    DEVICE_BAD_TABLE: "a table or index names rows outside the point array",
    DEVICE_TIMEOUT: "a bounded wait on a shared-memory bulk copy gave up",
    DEVICE_BATCH_RANGE: "a batch id lies outside [0, number of clouds)",
    DEVICE_NO_CANDIDATES: "a query has no candidate in its 27-cell neighbourhood",
    DEVICE_COPY_IN_FLIGHT: "a warp stopped while its bulk copies may still have been in flight",
}


class FknnError(RuntimeError):
    """Raised for any failure of the CUDA path (no silent fallback)."""


class FknnConfig(ctypes.Structure):
    _fields_ = [("warps_per_cta", ctypes.c_int32), ("tile_records", ctypes.c_int32),
                ("min_candidates_per_lane", ctypes.c_int32), ("ctas_per_sm", ctypes.c_int32),
                ("staging_depth", ctypes.c_int32)]

    def as_tuple(self):
        return (self.warps_per_cta, self.tile_records, self.min_candidates_per_lane,
                self.ctas_per_sm, self.staging_depth)


_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I32 = ctypes.c_int32
_F32 = ctypes.c_float
_SZ = ctypes.c_size_t

_SIGNATURES = {
    "fknn_version": (ctypes.c_char_p, []),
    "fknn_error_string": (ctypes.c_char_p, [ctypes.c_int]),
    "fknn_last_cuda_error": (ctypes.c_int, []),
    "fknn_read_status": (ctypes.c_int, [_P, _P, _P]),
    "fknn_read_candidate_stats": (ctypes.c_int, [_P, _P, _P, _P]),
    "fknn_last_launch_count": (ctypes.c_int, []),
    "fknn_profile_enable": (ctypes.c_int, [ctypes.c_int]),
    "fknn_profile_read": (ctypes.c_int, [_P, ctypes.c_int]),
    "fknn_workspace_bytes": (_SZ, [_I64, _I64, _I64, _I32]),
    "fknn_knn_offsets": (ctypes.c_int, [_P, _I64, _P, _I64, _P, _I64, _P, _I32, _F32, _I32,
                                        _F32, _P, _P, _P, _SZ, _P, _P]),
    "fknn_selftest_bounded_wait": (ctypes.c_int, [_P, _SZ, ctypes.c_uint32, _P]),
    "fknn_ball_query": (ctypes.c_int, [_P, _I64, _P, _I64, _P, _I64, _P, _I32, _F32, _I32, _F32,
                                       _P, _P, _P, _SZ, _P, _P]),
    "fknn_knn_grid": (ctypes.c_int, [_P, _P, _P, _I64, _P, _I64, _I32, _I32, _F32, _I32, _P, _P,
                                     _P, _SZ, _P, _P]),
    "fknn_tables_workspace_bytes": (_SZ, [_I64, _I64, _I64]),
    "fknn_query_tables": (ctypes.c_int, [_P, _I64, _P, _P, _P, _I64, _I32, _F32, _P, _P, _P, _SZ,
                                         _P, _P]),
    "fknn_query_tables_noalloc": (ctypes.c_int, [_P, _I64, _P, _P, _P, _I64, _I32, _F32, _P, _P,
                                                 _P]),
    "fknn_query_tables_noalloc_read_status": (ctypes.c_int, [_P, _P]),
    "fknn_general_query_tables": (ctypes.c_int, [_P, _I64, _P, _I64, _P, _P, _P, _P, _P, _I64,
                                                 _I32, _F32, _P, _P, _P, _SZ, _P, _P]),
    "fknn_selected_query_tables": (ctypes.c_int, [_P, _I64, _P, _I64, _P, _P, _P, _P, _I64, _I32,
                                                  _F32, _P, _P, _P, _SZ, _P, _P]),
    "fknn_morton_encode": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "fknn_morton_neighbor_keys": (ctypes.c_int, [_P, _P, _I64, _P, _P]),
    "fknn_build_tables_workspace_bytes": (_SZ, [_I64]),
    "fknn_build_tables": (ctypes.c_int, [_P, _P, _I64, _I32, _P, _P, _P, _P, _P, _P, _SZ, _P]),
    "fknn_backward_workspace_bytes": (_SZ, [_I64, _I64, _I32]),
    "fknn_backward": (ctypes.c_int, [_P, _I64, _P, _I64, _P, _P, _P, _I32, _P, _P, _I32, _P, _SZ,
                                     _P]),
    "fknn_back_query_workspace_bytes": (_SZ, [_I64, _I64]),
    "fknn_back_query": (ctypes.c_int, [_P, _I64, _P, _I64, _P, _F32, _I32, _I32, _P, _P, _P, _SZ,
                                       _P, _P]),
    "fknn_group_workspace_bytes": (_SZ, [_I64, _I32, _I64]),
    "fknn_group_features": (ctypes.c_int, [_P, _I64, _I32, _P, _I64, _I32, _P, _P, _I32, _P, _P,
                                           _SZ, _P]),
    "fknn_group_backward": (ctypes.c_int, [_P, _I64, _I32, _P, _I64, _I32, _I32, _P, _P, _I32, _P,
                                           _I32, _P, _SZ, _P]),
    "fknn_voxel_first_workspace_bytes": (_SZ, [_I64]),
    "fknn_voxel_first": (ctypes.c_int, [_P, _I64, _P, _F32, _P, _P, _P, _SZ, _P]),
    "fknn_adaptive_workspace_bytes": (_SZ, [_I64]),
    "fknn_adaptive_query": (ctypes.c_int, [_P, _P, _I64, _P, _I32, _I32, _I32, _I32, _F32, _I32,
                                           _P, _P, _P, _P, _SZ, _P, _P]),
}

EXPORTED = tuple(_SIGNATURES)

_lib = None
_lock = threading.Lock()


def load(path: str = LIB_PATH, require_cuda: bool = True):
    """Load libfknn.so once.  Raises FknnError if it is missing."""
    global _lib
    if require_cuda and not torch.cuda.is_available():
        raise FknnError("FlashKNN-B200 needs a CUDA device (sm_100a); none is visible")
    with _lock:
        if _lib is None:
            if not os.path.exists(path):
                raise FknnError(
                    f"{path} is missing: build it with `python -m flashknn_exprepo_b200.build`")
            lib = ctypes.CDLL(path)
            for name, (res, args) in _SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def load_for_inspection(path: str = LIB_PATH):
    """Load without requiring a GPU (symbol checks on CPU-only machines)."""
    return load(path, require_cuda=False)


def check(rc: int, what: str) -> None:
    if rc != FKNN_OK:
        lib = load_for_inspection()
        msg = lib.fknn_error_string(rc).decode()
        if rc == FKNN_ERR_CUDA:
            msg += f" (cudaError {lib.fknn_last_cuda_error()})"
        raise FknnError(f"{what}: {msg}")


def status_text(bits: int) -> str:
    return "; ".join(t for b, t in _STATUS_TEXT.items() if bits & b) or "ok"


def ptr(t) -> int | None:
    if t is None:
        return None
    return t.data_ptr()


def stream_handle(device=None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


class Workspace:
    """Scratch buffer per (host thread, device, stream), grown on demand
    (256-byte aligned).  Every host thread has its own buffers: two threads
    enqueueing on one stream at the same time would otherwise interleave
    their launches over one buffer.  A thread's buffers go with the thread."""

    def __init__(self):
        self._local = threading.local()

    def _bufs(self) -> dict:
        bufs = getattr(self._local, "bufs", None)
        if bufs is None:
            bufs = self._local.bufs = {}
        return bufs

    def get(self, nbytes: int, device: torch.device) -> torch.Tensor:
        key = (device.index, torch.cuda.current_stream(device).cuda_stream)
        bufs = self._bufs()
        buf = bufs.get(key)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
            bufs[key] = buf
        return buf

    def clear(self):
        """Drop the calling thread's buffers."""
        self._bufs().clear()


WORKSPACE = Workspace()


def read_status(ws: torch.Tensor) -> int:
    lib = load()
    out = ctypes.c_int(0)
    check(lib.fknn_read_status(ptr(ws), ctypes.byref(out), stream_handle(ws.device)),
          "fknn_read_status")
    return out.value


def candidate_stats(ws: torch.Tensor) -> tuple[int, int]:
    """(candidate total, groups) of the last self / general query that used
    ``ws`` (fknn_read_candidate_stats; synchronises the stream)."""
    lib = load()
    total, groups = ctypes.c_int64(0), ctypes.c_int64(0)
    check(lib.fknn_read_candidate_stats(ptr(ws), ctypes.byref(total), ctypes.byref(groups),
                                        stream_handle(ws.device)), "fknn_read_candidate_stats")
    return total.value, groups.value


def raise_on_status(ws: torch.Tensor, what: str, ignore: int = DEVICE_NO_CANDIDATES) -> None:
    """Raise FknnError for device status bits other than `ignore` (queries
    without candidates are valid for general queries: they are padded)."""
    bits = read_status(ws) & ~ignore
    if bits:
        raise FknnError(f"{what}: device reported {status_text(bits)} (status {bits})")
