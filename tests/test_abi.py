"""The C-ABI library loads and exports exactly the entry points include/mycel.h declares (no GPU needed)."""
import ctypes
import os
import re

import pytest

from mycel_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "mycel.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = set(re.findall(r"\b(mycel_[a-z0-9_]+)\s*\(", txt))
    return sorted(n for n in names if not n.endswith("_fn"))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "mycel_static_solve" in names and "mycel_simp_run" in names and "mycel_apply_k" in names
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert lib.mycel_version() >= 100


def test_context_without_device_fails_loudly():
    lib = _lib.load()
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    h = ctypes.c_void_p()
    st = lib.mycel_ctx_create(0, ctypes.byref(h))
    assert st == 7  # MYCEL_E_DEVICE
    assert b"CUDA" in lib.mycel_last_error(None)
    from mycel_b200 import api
    from mycel_b200.model import DeviceError
    with pytest.raises(DeviceError):
        api.Context(0)
