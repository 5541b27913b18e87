"""Golden fixtures of voxel-first subsampling and the DeLA hierarchy builder,
made by the reference's own ``Networks/hierarchy.py`` on CPU tensors.

Run this in a container that has the reference checkout (``oracle.build_ref.reference_root()``:
``FKNN_REFERENCE``, else the build container's mount point) after building the
oracle (``make -C oracle``).  The tests only read its outputs
(``hierarchy_<case>.npz``).

Stand-ins for what needs a GPU, as in the other generators here:
  * ``FlashKNN_Query_Dynamic_Load`` -> ``oracle.query_tables`` (restatement of
    that kernel, bit-exact against it on its table ABI);
  * ``FlashKNN_Nearest_Back_Query_DL`` / ``FlashKNN_Back_Query_DL`` ->
    ``oracle.back_query_tables``;
  * ``Tensor.argsort`` sorts stably.  The reference runs these sorts on CUDA
    tensors, where PyTorch's sort of more than 4096 keys is a stable radix
    sort; PyTorch's CPU argsort is not stable for small inputs.
Voxel sizes are powers of two, so ``xyz / size`` divides exactly and the CPU
run gives the cells of the CUDA run (where PyTorch multiplies by the FP32
reciprocal of the scalar).  The clouds hold no duplicate points, so no two
candidates tie in distance and the kernels' tie orders do not matter.
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

CASES = {
    # name: (points, voxel sizes, ks, alpha)
    "room_4levels_k8": (24000, (0.0625, 0.125, 0.25, 0.5), (8, 8, 8, 8), 16),
    "room_3levels_k16_alpha4": (16000, (0.03125, 0.125, 0.25), (16, 12, 8), 4),
}


def room_points(n, rng):
    """A noisy room (floor, ceiling, four walls, boxes), no duplicate points."""
    face = rng.integers(0, 6, n)
    u = rng.random(n)
    v = rng.random(n)
    dims = np.array([6.0, 8.0, 3.0])
    xyz = np.zeros((n, 3))
    for f in range(6):
        m = face == f
        ax = f // 2
        o1, o2 = [a for a in range(3) if a != ax]
        xyz[m, ax] = (f % 2) * dims[ax]
        xyz[m, o1] = u[m] * dims[o1]
        xyz[m, o2] = v[m] * dims[o2]
    xyz += rng.normal(0, 0.01, xyz.shape)
    xyz = xyz.astype(np.float32)
    _, first = np.unique(xyz, axis=0, return_index=True)
    return np.ascontiguousarray(xyz[np.sort(first)])


def main():
    torch.cuda.synchronize = lambda *a, **k: None  # CPU-only run
    functions = MG._import_reference(MG._Recorder())
    wrapper = sys.modules[functions.FlashKNN.__module__]

    def query(xyz, steps, neigh, cnt, k, out_idx, out_dis, bfp=8, cut_r2=float("inf")):
        idx, dist = O.query_tables(xyz.numpy(), steps.numpy(), neigh.numpy(), cnt.numpy(),
                                   int(k), cut_r2=np.float32(cut_r2))
        out_idx.copy_(torch.from_numpy(idx.astype(np.int32)))
        out_dis.copy_(torch.from_numpy(dist))

    def nearest(xyz_h, xyz_l, steps_h, steps_l, neigh, cnt, out_idx, out_dis):
        idx, dist = O.back_query_tables(xyz_h.numpy(), xyz_l.numpy(), steps_h.numpy(),
                                        steps_l.numpy(), neigh.numpy(), 1)
        out_idx.copy_(torch.from_numpy(idx.astype(np.int32)).reshape(out_idx.shape))
        out_dis.copy_(torch.from_numpy(dist).reshape(out_dis.shape))

    wrapper.FlashKNN_Query_Dynamic_Load = query
    wrapper.FlashKNN_Nearest_Back_Query_DL = nearest
    argsort = torch.Tensor.argsort
    torch.Tensor.argsort = lambda self, *a, **k: argsort(self, *a, **{**k, "stable": True})

    sys.path.insert(0, os.path.join(MG.REF, "Networks"))
    import hierarchy  # the reference's Networks/hierarchy.py

    for name, (n, sizes, ks, alpha) in CASES.items():
        rng = np.random.default_rng(SEED)
        xyz = room_points(n, rng)
        t = torch.from_numpy(xyz)
        vf = {f"voxel_first_{i}": hierarchy._voxel_first_cuda(t, s).numpy()
              for i, s in enumerate(sizes)}
        out = hierarchy.build_flash_hierarchy(t, sizes, ks, alpha)
        arrays = {f"ref_{i}": o.numpy() for i, o in enumerate(out)}
        np.savez_compressed(os.path.join(HERE, f"hierarchy_{name}.npz"), xyz=xyz,
                            voxel_sizes=np.asarray(sizes, np.float32), ks=np.asarray(ks),
                            alpha=np.int64(alpha), n_outputs=np.int64(len(out)), **vf, **arrays)
        print(name, len(xyz), "points;", [tuple(o.shape) for o in out])


if __name__ == "__main__":
    main()
