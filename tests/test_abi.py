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


def test_job_device_bytes_needs_no_device():
    """The admission estimate is host arithmetic: it grows with the grid and with the mixed workspace."""
    from mycel_b200 import api, workloads as W
    small = W.served_job(16, 8, 8, 2, seed=1, precision="fp64")
    big = W.served_job(32, 16, 16, 2, seed=1, precision="fp64")
    mixed = W.served_job(16, 8, 8, 2, seed=1, precision="mixed")
    b_small, b_big, b_mixed = (api.Server.device_bytes(m, o) for m, o in (small, big, mixed))
    assert 0 < b_small < b_big
    assert b_mixed > b_small
    # at least the problem's own FP64 vectors (F, b, diag, invD, 2 temporaries, 5 PCG vectors, u): 12 x 8 B/DOF
    assert b_small >= 12 * 8 * small[0].total_dofs
