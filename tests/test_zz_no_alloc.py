"""The OC update that allocates no device memory (mycel_oc_update_noalloc) against mycel_oc_update.

Callers that cannot allocate device memory when they run the OC step (their device memory is reserved by
another allocator, or they must not take the synchronisation of an allocation) pass their own device buffers;
the kernel's scratch lives in a fixed array inside the library. The inputs here sit in torch-owned device
memory, as they would in such a caller. Two calls in a row check that the shared array's leftover contents
from the first call do not leak into the second. Tolerance: the same as the other OC tests (bit-identical
densities and multiplier, since both entry points run the same kernel with the same grid).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    s = 0.5 + rng.random(n)
    pas = (rng.random(n) < 0.1).astype(np.uint8)
    rho = np.where(pas == 1, 1.0, rng.uniform(0.001, 1.0, n))
    dc = -10.0 ** (-3.0 + 8.0 * rng.random(n))
    return rho, dc, s, pas


def test_oc_update_noalloc_matches_oc_update():
    import torch
    from mycel_b200 import _lib, api
    ctx = api.default_context()
    lib = _lib.load()
    dev = torch.device("cuda", ctx.device)
    for n, seed, f in ((50_000, 1, 0.35), (7_001, 2, 0.2)):
        rho, dc, s, pas = _inputs(n, seed)
        ref, ref_lam = api.oc_update(rho, dc, s, pas, f, 0.2, 1e-3, 1.0, ctx=ctx)
        t_rho = torch.from_numpy(rho).to(dev)
        t_dc = torch.from_numpy(dc).to(dev)
        t_s = torch.from_numpy(s).to(dev)
        t_pas = torch.from_numpy(pas).to(dev)
        t_out = torch.full((n,), -1.0, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        lam = C.c_double(0.0)
        st = lib.mycel_oc_update_noalloc(ctx.handle, n, t_rho.data_ptr(), t_dc.data_ptr(), t_s.data_ptr(),
                                         t_pas.data_ptr(), t_out.data_ptr(), f, 0.2, 1e-3, 1.0, 60, 1e-8,
                                         C.byref(lam))
        assert st == 0, lib.mycel_last_error(ctx.handle)
        got = t_out.cpu().numpy()
        assert lam.value == ref_lam
        assert np.array_equal(got, ref)


def test_oc_update_noalloc_rejects_bad_arguments():
    from mycel_b200 import _lib, api
    ctx = api.default_context()
    lib = _lib.load()
    lam = C.c_double(0.0)
    st = lib.mycel_oc_update_noalloc(ctx.handle, -1, None, None, None, None, None, 0.3, 0.2, 1e-3, 1.0, 60, 1e-8,
                                     C.byref(lam))
    assert st == 1 and b"length" in lib.mycel_last_error(ctx.handle)


def test_oc_update_noalloc_other_call_forms():
    """No passive mask, the update written in place (rho_new == rho, as the SIMP loop calls it), n = 0, and a
    call repeated after a larger one: each equals mycel_oc_update, and the repeat gives the same bits as the
    first call with those inputs (nothing left in the shared array carries over)."""
    import torch
    from mycel_b200 import _lib, api
    ctx = api.default_context()
    lib = _lib.load()
    dev = torch.device("cuda", ctx.device)

    def call(rho, dc, s, pas, in_place):
        n = rho.size
        t_rho = torch.from_numpy(rho.copy()).to(dev)
        t_dc = torch.from_numpy(dc).to(dev)
        t_s = torch.from_numpy(s).to(dev)
        t_pas = None if pas is None else torch.from_numpy(pas).to(dev)
        t_out = t_rho if in_place else torch.full((n,), -1.0, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        lam = C.c_double(0.0)
        st = lib.mycel_oc_update_noalloc(ctx.handle, n, t_rho.data_ptr() if n else None,
                                         t_dc.data_ptr() if n else None, t_s.data_ptr() if n else None,
                                         None if t_pas is None or n == 0 else t_pas.data_ptr(),
                                         t_out.data_ptr() if n else None, 0.3, 0.2, 1e-3, 1.0, 60, 1e-8,
                                         C.byref(lam))
        assert st == 0, lib.mycel_last_error(ctx.handle)
        return t_out.cpu().numpy(), lam.value

    small = _inputs(9_000, 4)
    big = _inputs(60_000, 5)
    first = call(*small[:3], None, False)
    ref = api.oc_update(small[0], small[1], small[2], None, 0.3, 0.2, 1e-3, 1.0, ctx=ctx)
    assert first[1] == ref[1] and np.array_equal(first[0], ref[0])
    in_place = call(*small, True)
    ref = api.oc_update(*small, 0.3, 0.2, 1e-3, 1.0, ctx=ctx)
    assert in_place[1] == ref[1] and np.array_equal(in_place[0], ref[0])
    call(*big, False)
    again = call(*small[:3], None, False)
    assert again[1] == first[1] and np.array_equal(again[0], first[0])
    empty = np.zeros(0)
    _, lam0 = call(empty, empty, empty, None, False)
    assert lam0 == api.oc_update(empty, empty, empty, None, 0.3, 0.2, 1e-3, 1.0, ctx=ctx)[1]
