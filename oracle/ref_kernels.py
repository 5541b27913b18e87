"""Loader for the reference kernels built by oracle/build_ref.py (TEST ONLY)."""
from __future__ import annotations

import glob
import importlib.util
import os

HERE = os.path.dirname(os.path.abspath(__file__))
_mod = None


def path() -> str | None:
    hits = sorted(glob.glob(os.path.join(HERE, "_ref", "fknn_ref_cufun*.so")))
    return hits[0] if hits else None


def available() -> bool:
    return path() is not None


def load():
    global _mod
    if _mod is None:
        import torch  # noqa: F401  (libtorch symbols for the extension)
        p = path()
        if p is None:
            raise FileNotFoundError("oracle/_ref is empty: run `python oracle/build_ref.py`")
        spec = importlib.util.spec_from_file_location("fknn_ref_cufun", p)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _mod = mod
    return _mod
