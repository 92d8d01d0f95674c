"""The C-ABI library loads and exports every entry point include/steel_b200.h declares (CPU only)."""
import os
import re

from steel_webgpu_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "steel_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(steel_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol(steel):
    L = _lib.load()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.SIGNATURES), "binding and header disagree"


def test_no_device_is_reported_not_faked(steel):
    import ctypes
    import torch
    if torch.cuda.is_available():
        return
    L = _lib.load()
    p = ctypes.c_void_p()
    assert L.steel_ctx_create(0, ctypes.byref(p)) == 6  # STEEL_E_NODEVICE
    assert b"device" in L.steel_last_error()
