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


def _bisection_start(lam):
    # the bracket's two trials, then its expansions (lambda x 0.1 or x 10), then the bisection
    b = 2
    while b < len(lam) and (lam[b] == lam[b - 1] * 0.1 or lam[b] == lam[b - 1] * 10.0):
        b += 1
    return b


def _late_record_trial(lam, rels):
    # a late bisection trial whose relative error is below every earlier bisection trial's: with the tolerance
    # set to it, the reference stops exactly there
    b = _bisection_start(lam)
    for k in range(len(rels) - 1, b + 2, -1):
        if 0 < rels[k] < min(rels[b:k]):
            return k
    raise AssertionError("no record trial")


# f = 0.5: the target lies between the volumes at the largest and the smallest multiplier, so the bracket is
# found and the bisection runs
@pytest.mark.parametrize("n", [5000, 120_001, 1_769_472])
def test_tolerance_tie(oracle, ctx, n):
    rho, dc, s, pas = _inputs(n, 7 + n % 11)
    f = 0.5
    lam, vol, ts = oracle.oc_trace(rho, dc, s, pas, f, vol_tol=0.0)
    tv = f * ts
    rels = [_rel(v, tv) for v in vol]
    # the last record trial (relative error near 1e-16: decided in the last bits) and the first record below
    # 1e-7 (the range of the SIMP loop's 1e-8 tolerance)
    b = _bisection_start(lam)
    k_late = _late_record_trial(lam, rels)
    k_mid = next(k for k in range(b + 1, len(rels)) if rels[k] < 1e-7 and rels[k] < min(rels[b:k]))
    for k in (k_late, k_mid):
        for tol in (rels[k], float(np.nextafter(rels[k], 0.0)), float(np.nextafter(rels[k], 1.0))):
            oo, ol = oracle.oc_update(rho, dc, s, pas, f, 0.2, 1e-3, 1.0, 60, tol)
            go, gl = api.oc_update(rho, dc, s, pas, f, 0.2, 1e-3, 1.0, 60, tol, ctx=ctx)
            assert gl == ol, (k, tol)
            assert np.array_equal(go, oo)
        # at exactly the trial's relative error the reference stops on that trial
        assert oracle.oc_update(rho, dc, s, pas, f, 0.2, 1e-3, 1.0, 60, rels[k])[1] == lam[k]


@pytest.mark.parametrize("n", [5000, 120_001])
def test_equality_tie(oracle, ctx, n):
    # zero tolerance and a target equal to the reference's V(lambda) of a late bisection trial: the reference
    # stops there
    rho, dc, s, pas = _inputs(n, 3 + n % 7)
    lam, vol, ts = oracle.oc_trace(rho, dc, s, pas, 0.5, vol_tol=0.0)
    b = _bisection_start(lam)
    found = False
    for k in range(len(vol) - 1, b + 2, -1):
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
