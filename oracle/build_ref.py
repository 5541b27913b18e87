"""Compile the reference's own CUDA kernels for sm_100a into oracle/_ref/.

TEST INFRASTRUCTURE ONLY.  Run it in a container that has the reference
checkout (``reference_root()``: $FKNN_REFERENCE, else the build container's
mount point of the checkout); the built
module (oracle/_ref/fknn_ref_cufun*.so) is git-ignored and travels to the
GPU machine with the working tree.  It compiles the reference sources where
they lie -- FlashKNN/csrc/flash_knn_query_dynamic_load.cu (production SMPS
kernel, selected query, back query), flash_knn_query.cu and
flash_knn_construction.cu -- with the reference's own nvcc flags (-O2
-lineinfo) plus -gencode arch=compute_100a,code=sm_100a, and binds them with
oracle/ref_bindings.cpp.  The reference's setup.py is not used.

Load the result with ``oracle.ref_kernels.load()``.

``build_nanoflann`` compiles the reference's CPU kNN baseline -- nanoflann
over Query/ThirdParty/nanoflannkdtree/csrcs/nanoflann.hpp, with the
reference's flags (-O3 -mavx2 -funroll-loops) -- through the C binding
oracle/ref_nanoflann.cpp into oracle/_ref/libref_nanoflann.so (load it with
``oracle.ref_nanoflann``).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
NAME = "fknn_ref_cufun"
# where the build container mounts the reference checkout (read-only)
REFERENCE_MOUNT = "/root/reference"


def reference_root() -> str:
    """The reference checkout every recipe that reads the reference's
    sources uses: $FKNN_REFERENCE when set, else the build container's
    mount point.  The GPU machine has neither; nothing there calls this."""
    return os.environ.get("FKNN_REFERENCE") or REFERENCE_MOUNT


def build(reference: str | None = None, verbose: bool = False) -> str:
    reference = reference or reference_root()
    csrc = os.path.join(reference, "FlashKNN", "csrc")
    if not os.path.isdir(csrc):
        raise FileNotFoundError(f"reference sources not found under {csrc}")
    os.environ["TORCH_CUDA_ARCH_LIST"] = "10.0a"
    os.makedirs(OUT, exist_ok=True)
    from torch.utils.cpp_extension import load
    mod = load(
        name=NAME,
        sources=[os.path.join(csrc, "flash_knn_query_dynamic_load.cu"),
                 os.path.join(csrc, "flash_knn_query.cu"),
                 os.path.join(csrc, "flash_knn_construction.cu"),
                 os.path.join(HERE, "ref_bindings.cpp")],
        extra_include_paths=[csrc],
        extra_cflags=["-O3"],
        extra_cuda_cflags=["-O2", "-lineinfo"],
        build_directory=OUT,
        verbose=verbose,
        is_python_module=True,
    )
    return mod.__file__


def build_nanoflann(reference: str | None = None) -> str:
    reference = reference or reference_root()
    inc = os.path.join(reference, "Query", "ThirdParty", "nanoflannkdtree", "csrcs")
    if not os.path.isfile(os.path.join(inc, "nanoflann.hpp")):
        raise FileNotFoundError(f"nanoflann.hpp not found under {inc}")
    os.makedirs(OUT, exist_ok=True)
    out = os.path.join(OUT, "libref_nanoflann.so")
    subprocess.run(["g++", "-O3", "-mavx2", "-funroll-loops", "-fopenmp", "-fPIC", "-shared",
                    "-std=c++17", "-I", inc, os.path.join(HERE, "ref_nanoflann.cpp"), "-o", out],
                   check=True)
    return out


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
    print(build_nanoflann())
