"""Golden fixtures of the adaptive-neighbourhood query, made by the reference's
own code (``FlashKNN/functions/adaptive_octree.py``) on CPU tensors.

Run this in a container that has the reference checkout (``oracle.build_ref.reference_root()``:
``FKNN_REFERENCE``, else the build container's mount point) after building the
oracle (``make -C oracle``).  The tests only read its outputs
(``adaptive_<case>.npz``).

How the fixtures are made
-------------------------
``AdaptiveNeighborhoodFlashKNN.query`` runs unchanged except for four
stand-ins for what needs a GPU:
  * ``FlashKNN_Morton_Encode`` -> the reference's pure-torch encoder
    ``FlashKNN/functions/z_order.py:xyz2key`` (the same keys: checked by
    ``tests/test_oracle_golden.py`` against ``morton_keys.npz``);
  * ``FlashKNN_Morton_Neighbor_Keys`` -> ``xyz2key`` of the 27 offset
    coordinates, centre first, offsets (0, -1, +1)^3 in ij order
    (``FlashKNN/csrc/flash_knn_construction.cu:42-63``);
  * ``FlashKNN_Query_Dynamic_Load`` -> the oracle's restatement of that
    kernel (``oracle.query_tables``, bit-exact against the reference kernel
    on its table ABI), which fills the kernel's outputs so that the
    reference's own level selection, flattening and index remap produce the
    final answer;
  * the CUDA-tensor check of ``_validate_inputs`` is skipped (its other checks
    stay).
Saved per case: the inputs, the selected octree level of every point (in the
input order), and the reference's final int64 indices and FP32 distances.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import make_golden as MG  # noqa: E402
from oracle import oracle as O  # noqa: E402

SEED = MG.SEED

# name: (generator, voxel, K, min factor, max factor, max_shift or -1,
#        cut radius (inf = none), positions: "xyz" or "grid")
CASES = {
    "lidar_k16": ("lidar", 0.05, 16, 2, 8, -1, np.inf, "xyz"),
    "two_batches_k8": ("two_density", 0.05, 8, 2, 8, -1, np.inf, "xyz"),
    "room_k32_shift6": ("room", 0.04, 32, 2, 8, 6, np.inf, "xyz"),
    "lidar_grid_positions_k16": ("lidar", 0.05, 16, 2, 8, -1, np.inf, "grid"),
    "lidar_cut_k16_f1_4": ("lidar", 0.05, 16, 1, 4, -1, 1.5, "xyz"),
}


def make_adaptive_points(kind, voxel, rng):
    if kind == "lidar":
        rings, az = 16, 512
        elev = np.deg2rad(np.linspace(-24.8, 2.0, rings, dtype=np.float64))
        phi = np.linspace(0, 2 * np.pi, az, endpoint=False)
        e, p = np.meshgrid(elev, phi, indexing="ij")
        d = np.stack([np.cos(e) * np.cos(p), np.cos(e) * np.sin(p), np.sin(e)], -1).reshape(-1, 3)
        r = np.full(len(d), 30.0)
        down = d[:, 2] < -1e-6
        r[down] = np.minimum(1.7 / -d[down, 2], 30.0)         # ground at z = -1.7
        for _ in range(6):                                     # vertical cylinders
            cx, cy = rng.uniform(-20, 20, 2)
            rad = rng.uniform(0.3, 1.0)
            a = d[:, 0] ** 2 + d[:, 1] ** 2
            b = -2 * (d[:, 0] * cx + d[:, 1] * cy)
            c = cx * cx + cy * cy - rad * rad
            disc = b * b - 4 * a * c
            hit = disc > 0
            t = np.where(hit, (-b - np.sqrt(np.maximum(disc, 0))) / (2 * np.maximum(a, 1e-12)),
                         np.inf)
            ok = hit & (t > 0.5) & (t < r)
            r[ok] = t[ok]
        xyz = (d * r[:, None]).astype(np.float32)
        xyz += rng.normal(0, 0.01, xyz.shape).astype(np.float32)
        keep = rng.random(len(xyz)) > 0.1
        xyz = MG._dedup(xyz[keep].astype(np.float32), voxel, rng)
        return xyz, np.zeros(len(xyz), np.int64)
    if kind == "two_density":
        a = rng.random((2500, 3), dtype=np.float32) * np.float32(0.8)
        b = rng.random((700, 3), dtype=np.float32) * np.float32(6.0) - np.float32(3.0)
        a = MG._dedup(a, voxel, rng)
        b = MG._dedup(b, voxel, rng)
        xyz = np.concatenate([a, b]).astype(np.float32)
        batch = np.concatenate([np.zeros(len(a)), np.full(len(b), 2)]).astype(np.int64)
        return xyz, batch
    return MG.make_points(kind, voxel, rng)


def _stubs(functions):
    xyz2key = functions.xyz2key
    offsets = [(a, b, c) for a in (0, -1, 1) for b in (0, -1, 1) for c in (0, -1, 1)]

    def morton_encode(grid, batch):
        return xyz2key(grid[:, 0], grid[:, 1], grid[:, 2], batch)

    def neighbor_keys(coords, batch):
        out = torch.empty((coords.shape[0], 27), dtype=torch.int64)
        for j, (dx, dy, dz) in enumerate(offsets):
            out[:, j] = xyz2key(coords[:, 0] + dx, coords[:, 1] + dy, coords[:, 2] + dz, batch)
        return out.reshape(-1)

    def query(xyz, steps, neigh, cnt, k, out_idx, out_dis, bfp=1, cut_r2=float("inf")):
        idx, dist = O.query_tables(xyz.numpy(), steps.numpy(), neigh.numpy(), cnt.numpy(),
                                   int(k), cut_r2=np.float32(cut_r2))
        # rows past the query rows are the appended support copies: the
        # kernel iterates only over the query groups (neigh rows)
        m = out_idx.shape[0]
        out_idx.copy_(torch.from_numpy(idx[:m].astype(np.int32)))
        out_dis.copy_(torch.from_numpy(dist[:m]))

    return morton_encode, neighbor_keys, query


def main():
    torch.cuda.synchronize = lambda *a, **k: None  # CPU-only run
    functions = MG._import_reference(MG._Recorder())
    ao = sys.modules[functions.AdaptiveNeighborhoodFlashKNN.__module__]
    enc, nbr, query = _stubs(functions)
    ao.FlashKNN_Morton_Encode = enc
    ao.FlashKNN_Morton_Neighbor_Keys = nbr
    ao.FlashKNN_Query_Dynamic_Load = query
    original_validate = ao._validate_inputs

    def validate_cpu(grid_coord, batch_idx):
        # the reference's checks without the CUDA-tensor one
        if grid_coord.dtype != torch.int64 or batch_idx.dtype != torch.int64:
            raise ValueError("grid_coord and batch_idx must use torch.int64")
        if grid_coord.shape[0] == 0:
            raise ValueError("cannot construct an octree for an empty point cloud")
        if bool((batch_idx < 0).any()) or bool((batch_idx >= 32768).any()):
            raise ValueError("batch indices must lie in [0, 32768)")

    ao._validate_inputs = validate_cpu
    assert original_validate is not None

    for name, (kind, voxel, k, fmin, fmax, max_shift, cut, pos) in CASES.items():
        rng = np.random.default_rng(SEED)
        xyz, batch = make_adaptive_points(kind, voxel, rng)
        grid = np.floor(xyz / np.float32(voxel)).astype(np.int64)
        t_grid = torch.from_numpy(grid)
        t_batch = torch.from_numpy(batch)
        t_xyz = torch.from_numpy(xyz) if pos == "xyz" else None
        knn = functions.AdaptiveNeighborhoodFlashKNN(num_nbr=k, min_candidates_factor=fmin,
                                                     max_candidates_factor=fmax)
        shift = None if max_shift < 0 else max_shift
        idx, dist = knn.query(t_grid, t_batch, t_xyz, max_shift=shift, cut_radius=float(cut),
                              return_distances=True)
        hier = ao.build_adaptive_octree(t_grid, t_batch, shift)
        sel = ao.select_adaptive_levels(hier, k, fmin, fmax)
        levels = np.empty(len(xyz), np.int64)
        levels[hier.order.numpy()] = sel.numpy().astype(np.int64)
        stats = knn.last_stats
        np.savez_compressed(
            os.path.join(HERE, f"adaptive_{name}.npz"),
            xyz=xyz, grid=grid, batch=batch, k=np.int64(k), min_factor=np.int64(fmin),
            max_factor=np.int64(fmax), max_shift=np.int64(max_shift),
            cut_radius=np.float32(cut), grid_positions=np.bool_(pos == "grid"),
            ref_levels=levels, ref_idx=idx.numpy(), ref_dist=dist.numpy(),
            ref_level_node_counts=np.asarray(stats["level_node_counts"], np.int64))
        print(name, len(xyz), "points, levels", np.bincount(levels).tolist(),
              "octree levels", stats["octree_levels"])


if __name__ == "__main__":
    main()
