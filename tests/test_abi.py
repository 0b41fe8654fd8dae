"""The C-ABI library loads and exports every entry point include/fyzz_b200.h
declares (no device work: runs without a GPU)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "fyzz_b200.h")).read()
    return sorted(set(re.findall(r"\b(fyzz_b200_[a-z_0-9]+)\s*\(", text)))


def test_header_and_binding_agree(pkg):
    assert sorted(pkg.EXPORTS) == declared_symbols()


def test_library_exports_every_declared_symbol(pkg):
    if not os.path.exists(pkg.LIB_PATH):
        pkg.build()
    lib = ctypes.CDLL(pkg.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_create_without_device_fails_loudly(pkg):
    import torch
    if torch.cuda.is_available():
        return
    import pytest
    with pytest.raises(RuntimeError):
        pkg.World(0)
