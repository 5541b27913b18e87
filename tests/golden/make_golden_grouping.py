"""Golden fixtures of neighbour grouping, made by Pointcept's own
``pointops.grouping`` (``Pointcept/libs/pointops/functions/grouping.py:36-60``)
as shipped in the reference tree, on CPU tensors.

Run this in a container that has the reference checkout (``oracle.build_ref.reference_root()``:
``FKNN_REFERENCE``, else the build container's mount point).  The tests only read
its outputs (``grouping_<case>.npz``).

``grouping`` is plain torch indexing; only the module's import of the
compiled ``pointops._C`` (used by the other function in the file) is stubbed.
Saved per case: inputs, the grouped output and the gradients torch's
autograd gives for ``sum(grad_out * output)``.
"""
from __future__ import annotations

import importlib.util
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

# name: (n, m, k, c, with_xyz, separate queries)
CASES = {
    "feat16_self": (300, 300, 16, 16, False, False),
    "feat13_xyz_self": (300, 300, 8, 13, True, False),
    "feat32_xyz_queries": (400, 150, 12, 32, True, True),
}


def load_grouping():
    pkg = types.ModuleType("pointops")
    pkg.__path__ = []
    stub = types.ModuleType("pointops._C")
    stub.grouping_forward_cuda = stub.grouping_backward_cuda = None
    sys.modules["pointops"] = pkg
    sys.modules["pointops._C"] = stub
    path = os.path.join(REF, "Pointcept", "libs", "pointops", "functions", "grouping.py")
    spec = importlib.util.spec_from_file_location("pointops_grouping", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.grouping


def main():
    grouping = load_grouping()
    for name, (n, m, k, c, with_xyz, separate) in CASES.items():
        rng = np.random.default_rng(SEED)
        xyz = rng.random((n, 3), dtype=np.float32)
        feat = rng.standard_normal((n, c)).astype(np.float32)
        idx = rng.integers(0, n, (m, k)).astype(np.int32)
        idx[rng.random((m, k)) < 0.1] = -1          # padding entries
        idx[:5] = idx[0]                             # a few shared (hub) neighbours
        new_xyz = (rng.random((m, 3), dtype=np.float32) if separate else xyz)
        g_out = rng.standard_normal((m, k, c + (3 if with_xyz else 0))).astype(np.float32)
        t_xyz = torch.from_numpy(xyz).requires_grad_(True)
        t_new = torch.from_numpy(new_xyz.copy()).requires_grad_(True) if separate else t_xyz
        t_feat = torch.from_numpy(feat).requires_grad_(True)
        out = grouping(torch.from_numpy(idx), t_feat, t_xyz, t_new if separate else None,
                       with_xyz=with_xyz)
        (out * torch.from_numpy(g_out)).sum().backward()
        extra = {}
        if with_xyz:
            extra["ref_grad_xyz"] = t_xyz.grad.numpy()
            if separate:
                extra["ref_grad_new_xyz"] = t_new.grad.numpy()
        np.savez_compressed(os.path.join(HERE, f"grouping_{name}.npz"), xyz=xyz, feat=feat,
                            idx=idx, new_xyz=new_xyz, grad_out=g_out,
                            with_xyz=np.bool_(with_xyz), separate=np.bool_(separate),
                            ref_out=out.detach().numpy(), ref_grad_feat=t_feat.grad.numpy(),
                            **extra)
        print(name, tuple(out.shape))


if __name__ == "__main__":
    main()
