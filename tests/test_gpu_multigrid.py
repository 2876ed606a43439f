"""Multigrid forms against the FP64 oracle: MYCEL_PRECISION_FP64_MG ("mg", FP64 flexible CG on the factorised
operator preconditioned by an FP32 geometric multigrid V-cycle) and MYCEL_PRECISION_MIXED_MG ("mixed-mg", the same
iteration in FP32 inside FP64 iterative refinement).

Tolerances (stated): a solve to relative residual 1e-10 agrees with the oracle in u to 1e-7 of max|u| and
converges in the multigrid form itself (no fallback iterations) with at most a quarter of the oracle's Jacobi-PCG
iterations on grids of 8+ elements per axis; SIMP compliance within 1e-6 relative per iteration (solves to the
same residual tolerance as the oracle's).
"""
import numpy as np
import pytest

from mycel_b200 import api
from mycel_b200 import workloads as W
from models import carved_model, tiny_test_model

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def exact_oracle(oracle):
    oracle.set_modes(0, threads=8)
    yield
    oracle.set_modes(0)


# odd element counts (last coarse element of a single fine element), thin axes, carved domains
@pytest.mark.parametrize("prec", ["mg", "mixed-mg"])
@pytest.mark.parametrize("shape", [(31, 12, 9), (33, 17, 9), (40, 20, 10), (24, 6, 3), (5, 3, 2)])
def test_mg_solve_matches_oracle(oracle, ctx, shape, prec):
    m = carved_model(*shape, seed=8, emin_ratio=1e-9)
    om, pr = oracle.Model(m), api.Problem(m, ctx)
    b = om.forces() * (om.constrained() == 0)
    ref, rref = om.pcg_solve(b, tol=1e-10, max_iter=20000)
    u, r = pr.pcg_solve(b, tol=1e-10, max_iterations=20000, precision=prec)
    assert r.converged and r.final_residual <= 1e-10
    assert r.fallback_iterations == 0
    if min(shape) >= 8:
        assert r.iterations <= 0.25 * rref.iterations
    assert np.abs(u - ref).max() <= 1e-7 * np.abs(ref).max()


@pytest.mark.parametrize("prec", ["mg", "mixed-mg"])
def test_mg_grid_without_coarse_level_uses_fast_fp64(oracle, ctx, prec):
    m = tiny_test_model(1, 1, 1)
    om, pr = oracle.Model(m), api.Problem(m, ctx)
    b = om.forces() * (om.constrained() == 0)
    ref, _ = om.pcg_solve(b, tol=1e-10, max_iter=2000)
    u, r = pr.pcg_solve(b, tol=1e-10, max_iterations=2000, precision=prec)
    assert r.converged and r.inner_iterations == 0
    assert np.abs(u - ref).max() <= 1e-7 * np.abs(ref).max()


@pytest.mark.parametrize("prec", ["mg", "mixed-mg"])
def test_mg_warm_start_and_zero_rhs(oracle, ctx, prec):
    m = carved_model(20, 10, 8, seed=4)
    om, pr = oracle.Model(m), api.Problem(m, ctx)
    b = om.forces() * (om.constrained() == 0)
    u, r = pr.pcg_solve(b, tol=1e-9, max_iterations=5000, precision=prec)
    assert r.converged
    u2, r2 = pr.pcg_solve(b, tol=1e-9, max_iterations=5000, precision=prec, x0=u)
    assert r2.converged and r2.iterations == 0
    z, rz = pr.pcg_solve(np.zeros_like(b), tol=1e-9, max_iterations=5000, precision=prec)
    assert rz.converged and not z.any()


@pytest.mark.parametrize("prec", ["mg", "mixed-mg"])
def test_mg_simp_cantilever(oracle, ctx, prec):
    m, o = W.simp_cantilever_40x20x10()
    o = o.replace(max_iterations=8)
    ref = oracle.topopt_run(m, o)
    res = api.TopologyOptimizer.run(m, o.replace(precision=prec), ctx=ctx)
    assert res.total_iterations == ref.n_iters
    for a, b in zip(res.snapshots, ref.records):
        assert abs(a.compliance - b["compliance"]) <= 1e-6 * abs(b["compliance"])


@pytest.mark.parametrize("prec", ["mg", "mixed-mg"])
def test_mg_pitch_poisson_thin_plate_and_bridge(oracle, ctx, prec):
    """Voxel pitch h = 2.5 with nu = 0.28 (KE scaled and changed), a thin 48x40x2 plate (an axis that stops
    coarsening at one element), and a small bridge with corner supports: converged in the multigrid form itself,
    u within 1e-7 of the oracle's."""
    cases = [W.cantilever(24, 10, 6, h=2.5, nu=0.28, e0=1.0, emin_ratio=1e-9, force=-1.0),
             W.cantilever(48, 40, 2, e0=1.0, emin_ratio=1e-9, force=-1.0),
             W.bridge(48, 24, 24, support=4, load_patch=6)]
    for m in cases:
        om, pr = oracle.Model(m), api.Problem(m, ctx)
        b = om.forces() * (om.constrained() == 0)
        ref, rref = om.pcg_solve(b, tol=1e-10, max_iter=40000)
        u, r = pr.pcg_solve(b, tol=1e-10, max_iterations=40000, precision=prec)
        assert r.converged and r.final_residual <= 1e-10 and r.fallback_iterations == 0
        assert r.iterations < rref.iterations
        assert np.abs(u - ref).max() <= 1e-7 * np.abs(ref).max()
        pr.close()
