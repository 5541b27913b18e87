"""CPU: flashknn_exprepo_b200.cufun exports every name the reference wrapper
imports from its compiled module (FlashKnnWrapper.py:6-19), each taking the
positional arguments the reference declares (flash_knn_query.h,
flash_knn_construction.h).  Read as text from the reference checkout when it
is present; skipped otherwise."""
import inspect
import os
import re

import pytest

from oracle import build_ref


def _reference_file(*parts):
    path = os.path.join(build_ref.reference_root(), *parts)
    if not os.path.isfile(path):
        pytest.skip("the reference checkout is not present")
    return open(path, encoding="utf-8").read()


def test_module_exports_what_the_wrapper_imports():
    from flashknn_exprepo_b200 import cufun
    text = _reference_file("FlashKNN", "functions", "FlashKnnWrapper.py")
    block = re.search(r"from \.CuFun import \((.*?)\)", text, re.S).group(1)
    names = sorted(n.strip() for n in block.replace("\n", " ").split(",") if n.strip())
    assert names == sorted(cufun.__all__)


def test_positional_arity_follows_the_reference_declarations():
    from flashknn_exprepo_b200 import cufun
    decl = (_reference_file("FlashKNN", "csrc", "flash_knn_query.h")
            + _reference_file("FlashKNN", "csrc", "flash_knn_construction.h"))
    decl = re.sub(r"//[^\n]*", "", decl)  # comments hold commas too
    for name in cufun.__all__:
        if name == "get_cuda_shared_mem":
            continue
        m = re.search(rf"\b{name}\s*\(([^;{{]*?)\)\s*;", decl, re.S)
        assert m, name
        params = [p for p in m.group(1).split(",") if p.strip()]
        sig = inspect.signature(getattr(cufun, name))
        assert len(sig.parameters) == len(params), name
