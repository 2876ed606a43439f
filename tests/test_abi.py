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


def test_job_device_bytes_counts_the_multigrid_hierarchy():
    """The multigrid forms' estimate adds the hierarchy (coarse stencils, element matrices, vectors) to the
    mixed and fast FP64 workspaces; it scales with the grid."""
    from mycel_b200 import api, workloads as W
    est = {p: api.Server.device_bytes(*W.served_job(32, 16, 16, 2, seed=1, precision=p))
           for p in ("fp64", "mixed", "fp64f", "mg", "mixed-mg")}
    assert est["mixed-mg"] == est["mg"] > est["mixed"] > est["fp64"]
    assert est["mg"] > est["fp64f"]
    # level 1 of a 32x16x16 grid alone: 576 FP32 element-matrix entries per coarse element (16x8x8)
    assert est["mg"] - est["mixed"] >= 4 * 576 * 16 * 8 * 8
    big = api.Server.device_bytes(*W.served_job(64, 32, 32, 2, seed=1, precision="mg"))
    assert big > 6 * est["mg"]


def test_job_device_bytes_counts_separate_load_cases():
    """Load cases kept apart add each case's F, P F and u (3 x 8 B per DOF per case) to the estimate; with one
    load case the option changes nothing."""
    from mycel_b200 import api, workloads as W
    m, o = W.served_job(30, 14, 10, 2, seed=2, precision="mixed-mg")
    assert len(m.loads) == 3
    summed = api.Server.device_bytes(m, o)
    apart = api.Server.device_bytes(m, o.replace(separate_load_cases=True))
    assert apart - summed >= 3 * 8 * 3 * m.total_dofs
    m1, o1 = W.served_job(30, 14, 10, 2, seed=1, precision="mixed-mg")
    assert len(m1.loads) == 1
    assert api.Server.device_bytes(m1, o1) == api.Server.device_bytes(m1, o1.replace(separate_load_cases=True))
