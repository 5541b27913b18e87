"""FlashKNN-B200: grid k-nearest neighbours on sm_100a behind FlashKNN's API.

Public entry points (mirroring the reference's ``FlashKNN/functions``):
  FlashKNN              -- query / selected_query drop-in (wrapper.py)
  knn_query, KNNQuery   -- Pointcept-style offset batching with a
                           differentiable squared distance (pointops.py)
  knn_query_host        -- the same from host buffers to host buffers, copies
                           overlapped with the query cloud run by cloud run
  ball_query            -- radius-limited grid query, Pointcept's signature
  grouping, knn_query_and_group, ball_query_and_group
                        -- neighbour feature gather with a deterministic
                           backward (pointops.py)
  AdaptiveNeighborhoodFlashKNN
                        -- per-point octree level (adaptive.py)
  xyz2key               -- Morton keys (z_order.py)
  hierarchy             -- voxel-first subsampling and the DeLA hierarchy
                           builder (hierarchy.py)
  ops                   -- tensor-level C-ABI calls, incl. the reference
                           table ABI (query_tables, build_tables, ...)
The CUDA library is libfknn.so next to this file (``python -m
flashknn_exprepo_b200.build``); nothing falls back to the CPU.
"""
from . import hierarchy, ops
from ._lib import FknnError
from .adaptive import AdaptiveNeighborhoodFlashKNN
from .pointops import (KNNQuery, ball_query, ball_query_and_group, grouping, knn_query,
                       knn_query_and_group, knn_query_host)
from .wrapper import FlashKNN
from .z_order import xyz2key

__all__ = ["FlashKNN", "AdaptiveNeighborhoodFlashKNN", "KNNQuery", "knn_query", "knn_query_host",
           "ball_query",
           "grouping", "knn_query_and_group", "ball_query_and_group",
           "xyz2key",
           "hierarchy", "ops", "FknnError"]
