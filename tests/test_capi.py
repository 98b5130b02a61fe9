"""C-ABI library: builds for sm_100a, loads, and exports every declared symbol.

Runs without a GPU (no kernel is launched)."""

import ctypes
import os
import re
import shutil

import pytest

from conftest import REPO


def _declared_symbols():
    src = open(os.path.join(REPO, "include", "tsb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tsb_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def libpath():
    from tsb import build

    if shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"):
        if not os.path.exists(build.LIB_PATH):
            pytest.skip("no nvcc and no prebuilt libtsb.so")
        return build.LIB_PATH
    return build.build()


def test_header_declares_entry_points():
    syms = _declared_symbols()
    for s in ("tsb_nl_build", "tsb_pair_forward", "tsb_md_kick", "tsb_md_drift",
              "tsb_md_baoab_boa", "tsb_fused_md", "tsb_version"):
        assert s in syms


def test_library_exports_every_declared_symbol(libpath):
    lib = ctypes.CDLL(libpath)
    missing = [s for s in _declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_prototypes_cover_header(libpath):
    from tsb import _lib

    assert set(_lib.PROTOTYPES) == set(_declared_symbols())
    lib = _lib.load(libpath)
    assert lib.tsb_version().decode().startswith("tsb")
    assert lib.tsb_status_string(2).decode().startswith("capacity")


def test_workspace_sizes_without_gpu(libpath):
    from tsb import _lib

    lib = _lib.load(libpath)
    a = lib.tsb_nl_workspace_size(1000, 4)
    b = lib.tsb_nl_workspace_size(2000, 4)
    assert 0 < a < b
    assert lib.tsb_pair_workspace_size(1000, 4) > 0
    assert lib.tsb_fused_workspace_size(532000, 2048) > 0
    assert lib.tsb_fused_max_atoms() == 512


def test_ops_fail_loudly_without_cuda():
    import torch

    from tsb import _lib, neighbors

    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    pos = torch.zeros((2, 3), dtype=torch.float64)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        neighbors.torchsim_nl(pos, torch.eye(3, dtype=torch.float64), torch.ones(3, dtype=bool),
                              1.0, torch.zeros(2, dtype=torch.long))
    with pytest.raises(RuntimeError):
        _lib.require_cuda(pos)
