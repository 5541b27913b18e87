"""Golden fixtures of FlashKNN.back_query, made by the reference's own wrapper
(``FlashKNN/functions/FlashKnnWrapper.py:459-644``) on CPU tensors.

Run this in a container that has the reference checkout (``oracle.build_ref.reference_root()``:
``FKNN_REFERENCE``, else the build container's mount point) after building the
oracle (``make -C oracle``).  The tests only read its outputs
(``back_<case>.npz``).

CPU tensors take the wrapper's non-fused construction branch (``xyz2key``,
``argsort``, ``unique_consecutive``, ``torch.unique`` neighbour lookup).  The
two kernels it calls, ``FlashKNN_Nearest_Back_Query_DL`` (K = 1) and
``FlashKNN_Back_Query_DL`` (K > 1), are replaced by the oracle's restatement
over the same tables (``oracle.back_query_tables``); the wrapper's own
``order_l[out_indices[inverse_order]]`` remap produces the saved answer:
positions in ``sel_indices`` (and, for K > 1, squared distances).
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

# name: (generator, subset voxel, query grid size, K, batched).  The query
# grid sizes are powers of two: the wrapper's (xyz / size).long() divides
# exactly then, so the CPU run here and the reference's CUDA run (where
# PyTorch multiplies by the FP32 reciprocal of the scalar) give the same
# cells.
CASES = {
    "uniform_k1": ("uniform", 0.08, 0.125, 1, False),
    "uniform_k8": ("uniform", 0.08, 0.125, 8, False),
    "negative_two_batches_k4": ("negative", 0.1, 0.25, 4, True),
    "room_k16": ("room", 0.08, 0.25, 16, False),
}


def make_back_points(kind, rng):
    if kind == "uniform":
        return rng.random((3000, 3), dtype=np.float32), None
    if kind == "negative":
        a = (rng.random((1500, 3), dtype=np.float32) - np.float32(0.5)) * np.float32(2.4)
        b = (rng.random((1200, 3), dtype=np.float32) - np.float32(0.8)) * np.float32(1.5)
        xyz = np.concatenate([a, b]).astype(np.float32)
        batch = np.concatenate([np.zeros(1500), np.ones(1200)]).astype(np.int64)
        return xyz, batch
    if kind == "room":
        xyz, _ = MG.make_points("room", 0.02, rng)
        return xyz, None
    raise ValueError(kind)


def subset(xyz, batch, voxel):
    """First point of every occupied subset voxel (per batch), in input order."""
    g = np.floor(xyz / np.float32(voxel)).astype(np.int64)
    if batch is not None:
        g = np.concatenate([g, batch[:, None]], 1)
    _, first = np.unique(g, axis=0, return_index=True)
    return np.sort(first).astype(np.int64)


def main():
    torch.cuda.synchronize = lambda *a, **k: None  # CPU-only run
    functions = MG._import_reference(MG._Recorder())
    wrapper = sys.modules[functions.FlashKNN.__module__]

    def fill(xyz_h, xyz_l, steps_h, steps_l, neigh, k, out_idx, out_dis):
        idx, dist = O.back_query_tables(xyz_h.numpy(), xyz_l.numpy(), steps_h.numpy(),
                                        steps_l.numpy(), neigh.numpy(), k)
        out_idx.copy_(torch.from_numpy(idx.astype(np.int32)).reshape(out_idx.shape))
        out_dis.copy_(torch.from_numpy(dist).reshape(out_dis.shape))

    def nearest(xyz_h, xyz_l, steps_h, steps_l, neigh, cnt, out_idx, out_dis):
        fill(xyz_h, xyz_l, steps_h, steps_l, neigh, 1, out_idx, out_dis)

    def back(xyz_h, xyz_l, steps_h, steps_l, neigh, cnt, k, out_idx, out_dis):
        fill(xyz_h, xyz_l, steps_h, steps_l, neigh, int(k), out_idx, out_dis)

    wrapper.FlashKNN_Nearest_Back_Query_DL = nearest
    wrapper.FlashKNN_Back_Query_DL = back

    for name, (kind, voxel, size, k, batched) in CASES.items():
        rng = np.random.default_rng(SEED)
        xyz, batch = make_back_points(kind, rng)
        sel = subset(xyz, batch, voxel)
        knn = functions.FlashKNN(num_nbr=k)
        out = knn.back_query(torch.from_numpy(xyz), torch.from_numpy(sel), size, voxel,
                             None if batch is None else torch.from_numpy(batch))
        if k == 1:
            ref_idx, ref_dist = out.numpy(), np.zeros(0, np.float32)
        else:
            ref_idx, ref_dist = out[0].numpy(), out[1].numpy()
        np.savez_compressed(
            os.path.join(HERE, f"back_{name}.npz"), xyz=xyz, sel=sel,
            batch=np.zeros(0, np.int64) if batch is None else batch,
            query_grid_size=np.float32(size), k=np.int64(k), ref_idx=ref_idx, ref_dist=ref_dist)
        print(name, len(xyz), "points,", len(sel), "subset points")


if __name__ == "__main__":
    main()
