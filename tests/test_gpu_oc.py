"""OC update (OcOptimizer.Update, OcOptimizer.cs:12-175) on the device: near ties of the bisection and the
bounded grid-barrier waits.

The device sums V(lambda) as a tree; the reference sums in element order. Each decision (v < target,
v > target, relErr <= tolerance) is taken on the tree sum only when it lies farther from the threshold than
the tree sum's error bound, else on the sum in element order, so lambda and the densities are the
reference's bits. These tests build inputs whose threshold sits on one of the reference's own values.
"""
import numpy as np
import pytest

from mycel_b200 import api
from mycel_b200.model import TimeoutError_

pytestmark = pytest.mark.gpu


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    s = 0.5 + rng.random(n)
    pas = (rng.random(n) < 0.1).astype(np.uint8)
    rho = np.where(pas == 1, 1.0, rng.uniform(0.001, 1.0, n))
    dc = -10.0 ** (-3.0 + 8.0 * rng.random(n))
    return rho, dc, s, pas


def _rel(v, tv):
    return abs(v - tv) / max(tv, 1e-12)


def _late_record_trial(rels):
    # a late bisection trial whose relative error is below every earlier one's: with the tolerance set to it, the
    # reference stops exactly there
    k = len(rels) - 1
    while k > 0 and not (0 < rels[k] < min(rels[:k])):
        k -= 1
    assert k > 2
    return k


@pytest.mark.parametrize("n", [5000, 120_001, 1_769_472])
def test_tolerance_tie(oracle, ctx, n):
    rho, dc, s, pas = _inputs(n, 7 + n % 11)
    f = 0.35
    lam, vol, ts = oracle.oc_trace(rho, dc, s, pas, f, vol_tol=0.0)
    tv = f * ts
    rels = [_rel(v, tv) for v in vol]
    k = _late_record_trial(rels)
    for tol in (rels[k], float(np.nextafter(rels[k], 0.0)), float(np.nextafter(rels[k], 1.0))):
        oo, ol = oracle.oc_update(rho, dc, s, pas, f, 0.2, 1e-3, 1.0, 60, tol)
        go, gl = api.oc_update(rho, dc, s, pas, f, 0.2, 1e-3, 1.0, 60, tol, ctx=ctx)
        assert gl == ol, (k, tol)
        assert np.array_equal(go, oo)
    # at exactly the trial's relative error the reference stops on that trial
    assert oracle.oc_update(rho, dc, s, pas, f, 0.2, 1e-3, 1.0, 60, rels[k])[1] == lam[k]


@pytest.mark.parametrize("n", [5000, 120_001])
def test_equality_tie(oracle, ctx, n):
    # zero tolerance and a target equal to the reference's V(lambda) of a late trial: the reference stops there
    rho, dc, s, pas = _inputs(n, 3 + n % 7)
    lam, vol, ts = oracle.oc_trace(rho, dc, s, pas, 0.3, vol_tol=0.0)
    found = False
    for k in range(len(vol) - 1, 2, -1):
        f = vol[k] / ts
        for _ in range(8):
            if f * ts == vol[k]:
                break
            f = float(np.nextafter(f, np.inf if f * ts < vol[k] else -np.inf))
        if f * ts != vol[k]:
            continue
        lam2, vol2, _ = oracle.oc_trace(rho, dc, s, pas, f, vol_tol=0.0)
        if len(lam2) == k + 1 and lam2[k] == lam[k]:
            found = True
            break
    assert found
    oo, ol = oracle.oc_update(rho, dc, s, pas, f, 0.2, 1e-3, 1.0, 60, 0.0)
    go, gl = api.oc_update(rho, dc, s, pas, f, 0.2, 1e-3, 1.0, 60, 0.0, ctx=ctx)
    assert ol == lam[k] and gl == ol
    assert np.array_equal(go, oo)


def test_barrier_wait_runs_out_and_the_device_stays_usable(oracle):
    # every grid barrier waits for one block more than the grid has: each wait gives up after its poll limit, the
    # kernel returns and the call reports MYCEL_E_TIMEOUT; the next call on the same context works
    c = api.Context(0)
    try:
        rho, dc, s, pas = _inputs(20_000, 5)
        c.set_oc_wait(max_polls=20_000, unreachable=True)
        with pytest.raises(TimeoutError_):
            api.oc_update(rho, dc, s, pas, 0.35, ctx=c)
        c.set_oc_wait(0, False)
        go, gl = api.oc_update(rho, dc, s, pas, 0.35, ctx=c)
        oo, ol = oracle.oc_update(rho, dc, s, pas, 0.35)
        assert gl == ol and np.array_equal(go, oo)
    finally:
        c.close()
