"""CPU: the C-ABI library loads without a GPU and exports exactly the
declared entry points; the host-side API fails loudly without CUDA."""
import os
import re

import pytest
import torch

from flashknn_exprepo_b200 import _lib
from flashknn_exprepo_b200.build import build
from tests.conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "fknn.h")).read()
    return sorted(set(re.findall(r"FKNN_API\s+[\w\s\*]+?\b(fknn_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    build()
    return _lib.load_for_inspection()


def test_header_declares_the_binding_table():
    assert declared_symbols() == sorted(_lib.EXPORTED)


def test_library_exports_every_declared_symbol(lib):
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_library_exports_nothing_else():
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    names = sorted({ln.split()[-1] for ln in out.splitlines() if " T " in ln})
    assert names == declared_symbols()


def test_host_only_entry_points(lib):
    assert b"sm_100a" in lib.fknn_version()
    assert lib.fknn_error_string(_lib.FKNN_ERR_K).startswith(b"K must")
    # sizes are pure host arithmetic
    a = lib.fknn_workspace_bytes(1000, 1000, 1, _lib.QUERY_SELF)
    b = lib.fknn_workspace_bytes(2000, 2000, 1, _lib.QUERY_SELF)
    assert 0 < a < b
    assert lib.fknn_workspace_bytes(-1, 0, 1, 0) == 0
    assert lib.fknn_tables_workspace_bytes(100, 100, 10) > 0
    assert lib.fknn_backward_workspace_bytes(100, 100, 16) > 0


def test_argument_errors_return_before_any_launch(lib):
    # K outside [1, 64], null workspace, bad num_down: rejected on the host.
    assert lib.fknn_knn_offsets(None, 10, None, 1, None, 0, None, 65, 0.1, 2, 1.0, None, None,
                                None, 0, None, None) == _lib.FKNN_ERR_K
    assert lib.fknn_knn_offsets(None, 10, None, 1, None, 0, None, 16, 0.1, 2, 1.0, None, None,
                                None, 0, None, None) == _lib.FKNN_ERR_ARG
    assert lib.fknn_knn_grid(None, None, None, 10, None, 0, 16, 9, 1.0, 64, None, None, None, 0,
                             None, None) == _lib.FKNN_ERR_NUM_DOWN
    assert lib.fknn_query_tables(None, 10, None, None, None, 2, 0, 1.0, None, None, None, 0,
                                 None, None) == _lib.FKNN_ERR_K


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback():
    import flashknn_exprepo_b200 as fk
    xyz = torch.rand(100, 3)
    with pytest.raises(fk.FknnError):
        fk.knn_query(8, xyz, torch.tensor([100]), voxel_size=0.1)
    with pytest.raises(fk.FknnError):
        fk.FlashKNN(num_nbr=8).query(torch.zeros(100, 3, dtype=torch.long),
                                     torch.zeros(100, dtype=torch.long), xyz)
