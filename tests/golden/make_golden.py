"""Generate the golden fixtures in this directory from the reference's own code.

Run this in a container that has the reference checkout (``oracle.build_ref.reference_root()``:
``FKNN_REFERENCE``, else the build container's mount point).  It never runs on a
GPU machine and the tests only read its outputs (``*.npz``).

How the fixtures are made
-------------------------
* ``morton_keys.npz`` -- grid coordinates (including negative ones) and batch
  ids pushed through the reference's ``FlashKNN/functions/z_order.py:xyz2key``
  (pure torch, CPU).
* ``tables_<case>.npz`` -- the reference's ``FlashKNN.query`` and
  ``FlashKNN.selected_query`` (``FlashKNN/functions/FlashKnnWrapper.py``) run
  on CPU tensors.  CPU tensors take the wrapper's non-fused construction
  branch (``xyz2key`` + ``argsort`` + ``unique_consecutive`` + ``torch.unique``
  lookup, ``FlashKnnWrapper.py:231-337``).  The compiled kernel module
  ``CuFun`` is replaced by a stub that records the tables the wrapper hands
  to ``FlashKNN_Query_Dynamic_Load`` / ``FlashKNN_Selected_Query_DL``
  (sorted xyz, steps, neigh, cnt, query index, query steps), so the fixture
  holds exactly what the reference kernel would receive.

The reference kernel itself runs on these tables on the GPU in
``tests/test_gpu_parity.py`` (``test_reference_kernel_agrees_with_oracle``),
compiled for sm_100a by ``oracle/build_ref.py``; nothing kernel-made is
stored here.
"""
from __future__ import annotations

import importlib
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import build_ref  # noqa: E402

REF = build_ref.reference_root()
SEED = 47

CASES = {
    # name: (generator, voxel, num_down, K, selected stride or 0)
    "uniform_k16": ("uniform", 0.05, 2, 16, 0),
    "two_clouds_negative_k8": ("two_clouds", 0.05, 1, 8, 0),
    "uniform_selected_k16": ("uniform", 0.05, 2, 16, 3),
    "duplicate_voxels_k32": ("dups", 0.05, 2, 32, 0),
    "sparse_padding_k16": ("sparse", 0.05, 2, 16, 0),
    "dense_multibatch_k64": ("dense", 0.05, 1, 64, 0),
    "room_selected_k24": ("room", 0.04, 2, 24, 4),
}


def _dedup(xyz, voxel, rng):
    grid = np.floor(xyz / np.float32(voxel)).astype(np.int64)
    _, first = np.unique(grid, axis=0, return_index=True)
    keep = np.sort(first)
    return xyz[keep]


def make_points(kind, voxel, rng):
    """Small seeded clouds; returns (xyz f32 [n,3], batch int64 [n])."""
    if kind == "uniform":
        xyz = rng.random((2600, 3), dtype=np.float32)
        xyz = _dedup(xyz, voxel, rng)[:2000]
        return xyz, np.zeros(len(xyz), np.int64)
    if kind == "two_clouds":
        a = (rng.random((1800, 3), dtype=np.float32) - 0.5) * np.float32(1.2)
        b = (rng.random((1400, 3), dtype=np.float32) - 0.7) * np.float32(0.9)
        a = _dedup(a, voxel, rng)
        b = _dedup(b, voxel, rng)
        xyz = np.concatenate([a, b]).astype(np.float32)
        batch = np.concatenate([np.zeros(len(a)), np.ones(len(b))]).astype(np.int64)
        return xyz, batch
    if kind == "dups":
        xyz = rng.random((1500, 3), dtype=np.float32) * np.float32(0.6)
        return xyz, np.zeros(len(xyz), np.int64)
    if kind == "sparse":
        xyz = rng.random((300, 3), dtype=np.float32) * np.float32(40.0)
        xyz = np.concatenate([xyz, xyz[:40] + np.float32(0.01)]).astype(np.float32)
        xyz = _dedup(xyz, voxel, rng)
        return xyz, np.zeros(len(xyz), np.int64)
    if kind == "dense":
        clouds, batches = [], []
        for c in range(3):
            pts = rng.random((1200, 3), dtype=np.float32) * np.float32(0.45) + np.float32(c * 0.3)
            pts = _dedup(pts, voxel, rng)
            clouds.append(pts)
            batches.append(np.full(len(pts), c, np.int64))
        return np.concatenate(clouds).astype(np.float32), np.concatenate(batches)
    if kind == "room":
        n = 4000
        face = rng.integers(0, 6, n)
        u = rng.random(n, dtype=np.float32)
        v = rng.random(n, dtype=np.float32)
        dims = np.array([1.2, 1.6, 0.8], np.float32)
        xyz = np.zeros((n, 3), np.float32)
        for f in range(6):
            m = face == f
            ax = f // 2
            o1, o2 = [a for a in range(3) if a != ax]
            xyz[m, ax] = (f % 2) * dims[ax]
            xyz[m, o1] = u[m] * dims[o1]
            xyz[m, o2] = v[m] * dims[o2]
        xyz += rng.normal(0, 0.005, xyz.shape).astype(np.float32)
        xyz -= xyz.min(0)
        xyz = _dedup(xyz.astype(np.float32), voxel, rng)
        return xyz, np.zeros(len(xyz), np.int64)
    raise ValueError(kind)


class _Recorder:
    def __init__(self):
        self.calls = []

    def query(self, xyz, steps, neigh, cnt, k, out_idx, out_dis, bfp=8, cut_r2=float("inf")):
        self.calls.append(dict(kind="query", xyz_sorted=xyz.clone(), steps=steps.clone(),
                               neigh=neigh.clone(), cnt=cnt.clone(), k=int(k),
                               cut_r2=float(cut_r2)))

    def selected(self, xyz, qindex, steps, steps_query, neigh, cnt, k, out_idx, out_dis,
                 bfp=8, cut_r2=float("inf")):
        self.calls.append(dict(kind="selected", xyz_sorted=xyz.clone(), qindex=qindex.clone(),
                               steps=steps.clone(), steps_query=steps_query.clone(),
                               neigh=neigh.clone(), cnt=cnt.clone(), k=int(k),
                               cut_r2=float(cut_r2)))


def _import_reference(recorder):
    stub = types.ModuleType("functions.CuFun")

    def unavailable(*_a, **_k):
        raise RuntimeError("kernel stub: not part of the table capture")

    for name in ("FlashKNN_Back_Query_DL", "FlashKNN_Morton_Encode",
                 "FlashKNN_Morton_Neighbor_Keys", "FlashKNN_Nearest_Back_Query_DL",
                 "FlashKNN_Query_Dynamic_Load_Ablation",
                 "FlashKNN_Query_Dynamic_Load_Thread_Group", "FlashKNN_Query_GM",
                 "FlashKNN_Query_GMPS", "FlashKNN_Query_SMSS"):
        setattr(stub, name, unavailable)
    stub.get_cuda_shared_mem = lambda: 49152
    stub.FlashKNN_Query_Dynamic_Load = recorder.query
    stub.FlashKNN_Selected_Query_DL = recorder.selected
    sys.modules["functions.CuFun"] = stub
    sys.path.insert(0, os.path.join(REF, "FlashKNN"))
    functions = importlib.import_module("functions")
    return functions


def main():
    torch.cuda.synchronize = lambda *a, **k: None  # CPU-only capture
    recorder = _Recorder()
    functions = _import_reference(recorder)
    FlashKNN = functions.FlashKNN
    xyz2key = functions.xyz2key

    # --- morton keys from the reference's LUT encoder
    rng = np.random.default_rng(SEED)
    g = rng.integers(-2**15, 2**15, size=(4096, 3), dtype=np.int64)
    g[:8] = [[0, 0, 0], [-1, -1, -1], [1, 2, 3], [-2**15, 2**15 - 1, 0],
             [255, 256, -256], [12345, -12345, 7], [2**15 - 1, 2**15 - 1, 2**15 - 1],
             [-2**15, -2**15, -2**15]]
    b = rng.integers(0, 2**15, size=4096, dtype=np.int64)
    keys = xyz2key(torch.from_numpy(g[:, 0]), torch.from_numpy(g[:, 1]),
                   torch.from_numpy(g[:, 2]), torch.from_numpy(b)).numpy()
    keys_nob = xyz2key(torch.from_numpy(g[:, 0]), torch.from_numpy(g[:, 1]),
                       torch.from_numpy(g[:, 2])).numpy()
    np.savez_compressed(os.path.join(HERE, "morton_keys.npz"), grid=g, batch=b, keys=keys,
                        keys_nobatch=keys_nob)

    # --- reference tables
    for name, (kind, voxel, num_down, k, stride) in CASES.items():
        rng = np.random.default_rng(SEED)
        xyz, batch = make_points(kind, voxel, rng)
        grid = np.floor(xyz / np.float32(voxel)).astype(np.int64)
        t_xyz = torch.from_numpy(xyz)
        t_grid = torch.from_numpy(grid)
        t_batch = torch.from_numpy(batch)
        flash = FlashKNN(num_nbr=k, num_down=num_down)
        recorder.calls.clear()
        if stride:
            qidx = np.arange(0, len(xyz), stride, dtype=np.int64)
            flash.selected_query(t_xyz, t_grid, torch.from_numpy(qidx), t_batch,
                                 memory_mode="SM")
        else:
            qidx = np.zeros(0, np.int64)
            flash.query(t_grid, t_batch, t_xyz, memory_mode="SM", sorting_mode="PS")
        (call,) = recorder.calls
        out = dict(xyz=xyz, grid=grid, batch=batch, voxel=np.float32(voxel),
                   num_down=np.int64(num_down), k=np.int64(k), query_indices=qidx)
        for key, val in call.items():
            if isinstance(val, torch.Tensor):
                out["ref_" + key] = val.numpy()
        np.savez_compressed(os.path.join(HERE, f"tables_{name}.npz"), **out)
        print(name, len(xyz), "points,", call["neigh"].shape[0], "parents")


if __name__ == "__main__":
    main()
