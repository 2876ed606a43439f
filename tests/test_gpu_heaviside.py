"""HeavisideProjection (HeavisideProjection.cs:12-37) on the device against the oracle, and a SIMP run with
EnableHeaviside (TopologyOptimizer.cs:192-199, 279-290, beta doubling :315-318) against the oracle's run.

The expressions are the reference's, rounded per operation; tanh is CUDA's, not the C library's, so values
may differ in the last bits: projections and derivatives are held to 4e-16 absolute (a few ulp of values in
[0, beta]). Those last bits move the SIMP trajectory a little (2.4e-8 relative in compliance by iteration 22 on
the cantilever below): the run is held to 1e-6 relative in compliance per iteration and 1e-4 in the final
densities."""
import numpy as np
import pytest

from mycel_b200 import api, workloads as W
from mycel_b200.model import OptimizerOptions

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("beta", [1.0, 2.0, 4.0, 8.0])
def test_project_and_derivative(oracle, ctx, beta):
    rng = np.random.default_rng(int(beta))
    rt = np.concatenate([rng.random(200_000), [0.0, 0.5, 1.0, 1e-3, 1 - 1e-12]])
    p = api.HeavisideProjection.project(rt, beta, ctx=ctx)
    d = api.HeavisideProjection.derivative(rt, beta, ctx=ctx)
    assert np.abs(p - oracle.heaviside_project(rt, beta)).max() <= 4e-16
    assert np.abs(d - oracle.heaviside_derivative(rt, beta)).max() <= 4e-16 * beta
    assert p.min() >= 0.0 and p.max() <= 1.0 and d.min() >= 1e-12


def test_nan_semantics(oracle, ctx):
    # Math.Clamp lets NaN through (Project) and Math.Max(NaN, 1e-12) is NaN (Derivative)
    rt = np.array([np.nan, 0.25])
    assert np.isnan(api.HeavisideProjection.project(rt, 2.0, ctx=ctx)[0])
    assert np.isnan(api.HeavisideProjection.derivative(rt, 2.0, ctx=ctx)[0])
    assert np.isnan(oracle.heaviside_derivative(rt, 2.0)[0])


def test_simp_with_heaviside(oracle, ctx):
    m = W.cantilever(20, 8, 4, e0=1.0, emin_ratio=1e-9, force=-1.0)
    o = OptimizerOptions(volume_fraction=0.35, filter_radius_mm=1.5, max_iterations=30, enable_heaviside=True,
                         solver_tolerance_initial=1e-8, solver_tolerance_final=1e-8)
    ref = oracle.topopt_run(m, o)
    res = api.TopologyOptimizer.run(m, o, ctx=ctx)
    assert res.total_iterations == ref.n_iters == 30  # beta doubles at iteration 25
    for a, b in zip(res.snapshots, ref.records):
        assert abs(a.compliance - b["compliance"]) <= 1e-6 * abs(b["compliance"])
    assert np.abs(res.final_physical_density - ref.phys).max() <= 1e-4
