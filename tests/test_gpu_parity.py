"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Bar: bit-exact for the plain FP64 path (same operation order, no FMA). The oracle runs with its integer-power
switch on (correctly rounded rho^p, which is what the kernels compute; see oracle.h), and with the default
Vector256.Sum lane order (lane mode 0).
"""
import numpy as np
import pytest

from mycel_b200 import api
from mycel_b200 import workloads as W
from mycel_b200.model import (ArgumentError, FeMaterial, FeModel, GridSpec, InvalidOperationError, LoadCase,
                              OptimizerOptions, StaticAnalysisOptions, SurfacePatch)
from models import bar_model, carved_model, l_shape_domain, tiny_test_model, underconstrained_model

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def exact_oracle(oracle):
    oracle.set_modes(lane_mode=0, threads=8)
    yield
    oracle.set_modes(0)


GRIDS = [(1, 1, 1), (2, 3, 5), (7, 4, 3), (40, 20, 10), (33, 17, 9)]


@pytest.mark.parametrize("shape", GRIDS)
def test_matvec_fp64_bit_exact(oracle, ctx, shape):
    nx, ny, nz = shape
    m = carved_model(nx, ny, nz, seed=nx, frac=0.15) if nx > 2 else tiny_test_model(nx, ny, nz)
    om = oracle.Model(m)
    pr = api.Problem(m, ctx)
    x = np.random.default_rng(1).uniform(-1, 1, m.total_dofs)
    assert np.array_equal(pr.apply_k(x), om.apply_k(x))
    xp = x * (om.constrained() == 0)
    assert np.array_equal(pr.apply_k(xp, projected=True), om.apply_a(xp, projected=True))
    assert np.array_equal(pr.diagonal(), om.diag())


def test_matvec_density_update_and_h(oracle, ctx):
    m = carved_model(12, 6, 5, seed=9)
    g = GridSpec(12, 6, 5, 2.5)
    m2 = FeModel(g, m.domain, FeMaterial(3000.0, 0.28, 1e-6), m.fixed_dofs, m.loads, m.element_density, 3.0)
    om = oracle.Model(m2)
    pr = api.Problem(m2, ctx)
    d = np.random.default_rng(5).uniform(0.001, 1.0, g.total_elements)
    om.update_densities(d, 3.0)
    pr.update_densities(d, 3.0)
    x = np.random.default_rng(2).normal(size=m2.total_dofs)
    assert np.array_equal(pr.apply_k(x), om.apply_k(x))
    assert np.array_equal(pr.diagonal(), om.diag())


@pytest.mark.parametrize("lane", [1, 2])
def test_lane_modes_change_bits_not_values(oracle, ctx, lane):
    # the lane-combine switch only moves the last bits: the CUDA default (mode 0) stays within 1e-14
    m = carved_model(10, 6, 4, seed=4)
    x = np.random.default_rng(3).normal(size=m.total_dofs)
    y0 = api.Problem(m, ctx).apply_k(x)
    oracle.set_modes(lane)
    y1 = oracle.Model(m).apply_k(x)
    assert np.abs(y0 - y1).max() <= 1e-14 * np.abs(y1).max()


def test_pcg_solve_bit_exact(oracle, ctx):
    m = tiny_test_model()
    om = oracle.Model(m)
    pr = api.Problem(m, ctx)
    b = om.forces() * (om.constrained() == 0)
    ug, rg = pr.pcg_solve(b, tol=1e-10, max_iterations=5000)
    uo, ro = om.pcg_solve(b, tol=1e-10, max_iter=5000)
    assert rg.iterations == ro.iterations and rg.converged and ro.converged
    assert rg.final_residual == ro.final_residual
    assert np.array_equal(ug, uo)
    # warm start from a perturbed solution
    x0 = uo * 0.9
    ug2, rg2 = pr.pcg_solve(b, x0=x0, tol=1e-10)
    uo2, ro2 = om.pcg_solve(b, x0=x0, tol=1e-10)
    assert rg2.iterations == ro2.iterations and np.array_equal(ug2, uo2)


def test_pcg_unprojected_rhs_and_max_iterations(oracle, ctx):
    g = GridSpec(4, 2, 2, 1.0)
    fixed = FeModel.fix_dofs([g.node_index(0, j, k) for k in range(3) for j in range(3)])
    m = FeModel(g, np.ones(16), FeMaterial(1000.0, 0.3), fixed)
    pr, om = api.Problem(m, ctx), oracle.Model(m)
    b = np.zeros(m.total_dofs)
    b[3 * g.node_index(4, 1, 1) + 2] = -50.0
    b[fixed] = 12345.67
    ug, rg = pr.pcg_solve(b, tol=1e-6)
    uo, ro = om.pcg_solve(b, tol=1e-6)
    assert np.array_equal(ug, uo) and np.all(ug[fixed] == 0.0)
    ug, rg = pr.pcg_solve(b, tol=1e-12, max_iterations=3)
    uo, ro = om.pcg_solve(b, tol=1e-12, max_iter=3)
    assert not rg.converged and rg.iterations == 3 and rg.message == ro.message
    assert np.array_equal(ug, uo)
    ug, rg = pr.pcg_solve(np.zeros(m.total_dofs), x0=np.ones(m.total_dofs))
    assert rg.converged and rg.message == "RHS is zero. Solution is zero." and not ug.any()


def test_static_solve_parity(oracle, ctx):
    model, tip = bar_model(40.0, 10.0, 10.0, 2.5, 3000.0, 0.3)
    model.loads.append(LoadCase(tip, (500.0, -200.0, -800.0)))
    g = api.StaticAnalysis.run(model, StaticAnalysisOptions(tolerance=1e-8), ctx)
    o = oracle.static_run(model, 1e-8, 5000)
    assert g.solver_info.iterations == o.solver_info.iterations
    assert np.array_equal(g.u, o.u)
    assert g.compliance == o.compliance and g.max_displacement == o.max_displacement
    assert np.array_equal(g.reactions, o.reactions)
    vm = oracle.Model(model).von_mises(o.u)
    assert np.array_equal(g.von_mises_per_element, vm)


def test_static_errors_match_reference(ctx):
    with pytest.raises(InvalidOperationError, match="(?i)sufficiently constrained"):
        api.StaticAnalysis.run(underconstrained_model(), StaticAnalysisOptions(1e-6, 500), ctx)
    g = GridSpec(2, 2, 2, 1.0)
    m = FeModel(g, np.ones(8), FeMaterial(1000.0, 0.3), FeModel.fix_dofs([0, 1]))
    with pytest.raises(ArgumentError):
        api.StaticAnalysis.run(m, StaticAnalysisOptions(warm_start_displacements=np.zeros(m.total_dofs - 1)), ctx)
    m = FeModel(g, np.ones(8), FeMaterial(1000.0, 0.3), [0, 1, 2], [LoadCase(SurfacePatch([26], [1.0]), (0, 0, -1))])
    with pytest.raises(InvalidOperationError, match="fewer than 6"):
        api.StaticAnalysis.run(m, None, ctx)


@pytest.mark.parametrize("rmin,shape", [(1.5, (9, 7, 6)), (1.8, (9, 7, 6)), (2.5, (9, 7, 6)), (3.0, (9, 7, 6)),
                                        (2.5, (70, 19, 9)), (4.2, (37, 12, 11)), (8.5, (30, 12, 10))])
def test_filter_bit_exact(oracle, ctx, rmin, shape):
    """Shared-memory tiles (several tiles and partial ones; rmin 8.5 exceeds the tile limit and runs the
    per-element kernel): the same bits as the oracle."""
    g, dom = l_shape_domain(*shape)
    act = np.nonzero(dom)[0].astype(np.int32)
    m = FeModel(g, dom, FeMaterial(1.0, 0.3), FeModel.fix_dofs(range(3)))
    pr = api.Problem(m, ctx)
    fg = api.DensityFilter(pr, rmin)
    fo = oracle.Filter(g, dom, act, rmin)
    x = np.random.default_rng(7).random(act.size)
    assert np.array_equal(fg.s, fo.s)
    assert np.array_equal(fg.apply(x), fo.apply(x))
    assert np.array_equal(fg.adjoint(x), fo.adjoint(x))


def test_sensitivities_bit_exact(oracle, ctx):
    m = carved_model(11, 5, 4, seed=2)
    om, pr = oracle.Model(m), api.Problem(m, ctx)
    u = np.random.default_rng(11).normal(size=m.total_dofs)
    rho = np.random.default_rng(12).uniform(0.001, 1.0, m.active_element_count)
    assert np.array_equal(pr.sensitivities(u, rho, 3.0), om.sensitivities(u, rho, 3.0))


@pytest.mark.parametrize("n", [0, 1, 200, 5000, 120_001, 1_769_472])
def test_oc_update_matches(oracle, ctx, n):
    rng = np.random.default_rng(n + 5)
    s = 0.5 + rng.random(n)
    pas = (rng.random(n) < 0.1).astype(np.uint8)
    rho = np.where(pas == 1, 1.0, rng.uniform(0.001, 1.0, n))
    dc = -10.0 ** (-3.0 + 8.0 * rng.random(n))
    if n:
        dc[rng.integers(0, n, max(1, n // 50))] = 0.0
    for lg in (1.0, 1e-30, float("nan")):
        go, gl = api.oc_update(rho, dc, s, pas, 0.35, 0.2, 1e-3, lg, ctx=ctx)
        oo, ol = oracle.oc_update(rho, dc, s, pas, 0.35, 0.2, 1e-3, lg)
        # the volume sums are reduced as a tree on the device; every bisection decision is still the sequential
        # sum's (near ties are settled by the sum in element order)
        assert gl == ol
        assert np.array_equal(go, oo)


def test_simp_cantilever_40x20x10_parity(oracle, ctx):
    """SIMP cantilever 40x20x10 (8,000 elements), FP64 plain path vs oracle, reference defaults (hinges on)."""
    m, o = W.simp_cantilever_40x20x10()
    ref = oracle.topopt_run(m, o)
    res = api.TopologyOptimizer.run(m, o, ctx=ctx)
    assert res.total_iterations == ref.n_iters
    for a, b in zip(res.snapshots, ref.records):
        assert a.solver_iterations == b["solver_iterations"]
        assert abs(a.compliance - b["compliance"]) <= 1e-10 * abs(b["compliance"])
        assert abs(a.volume_fraction - b["volume_fraction"]) <= 1e-12
        assert a.max_change == b["max_change"]
    assert np.abs(res.final_displacements - ref.u).max() <= 1e-10 * np.abs(ref.u).max()
    assert np.array_equal(res.final_physical_density, ref.phys)
    assert np.array_equal(res.final_design_density, ref.design)


def test_simp_options_paths(oracle, ctx):
    """Continuation, passive mask, no hinges, initial density and warm start go through the same logic."""
    m = W.cantilever(16, 6, 4)
    pm = np.zeros(m.total_elements, np.uint8)
    pm[::17] = 1
    init = np.random.default_rng(3).uniform(0.2, 0.6, m.total_elements).astype(np.float32)
    o = OptimizerOptions(volume_fraction=0.35, filter_radius_mm=1.2, max_iterations=6, continuation=True,
                         passive_mask=pm, initial_density=init, protect_boundary_hinges=False,
                         solver_tolerance_initial=1e-6, solver_tolerance_final=1e-8)
    ref = oracle.topopt_run(m, o)
    res = api.TopologyOptimizer.run(m, o, ctx=ctx)
    assert [s.solver_iterations for s in res.snapshots] == [r["solver_iterations"] for r in ref.records]
    assert np.array_equal(res.final_physical_density, ref.phys)


@pytest.mark.parametrize("p", [1.0, 2.0, 3.0, 3.5])
def test_device_pow_bit_exact(oracle, ctx, p):
    # Math.Pow on the device (E_e: rho^p, FemOperator.cs:100,133; sensitivities: rho^(p-1),
    # SensitivityAnalysis.cs:93-95) carries the C library's bits: 10^7 densities in [1e-9, 1] at p and p - 1
    rng = np.random.default_rng(int(10 * p))
    x = 1e-9 + rng.random(10_000_000) * (1 - 1e-9)
    for y in (p, p - 1.0):
        d = api.math_pow(x, y, ctx)
        h = oracle.math_pow(x, y)
        assert np.array_equal(d.view(np.uint64), h.view(np.uint64)), (p, y)


def test_device_pow_wide_range_bit_exact(oracle, ctx):
    rng = np.random.default_rng(9)
    n = 2_000_000
    x = np.ldexp(rng.random(n) + 0.5, rng.integers(-1074, 1024, n))
    y = rng.uniform(-60, 60, n)
    with np.errstate(all="ignore"):
        for xs, ys in ((x, y), (-x, np.floor(y)), (rng.uniform(1e-3, 0.5, n), rng.uniform(-1075, -700, n))):
            if ys.max() < -600:
                ys = ys / np.log(xs)
            d = api.math_pow(xs, ys, ctx)
            h = oracle.math_pow(xs, ys)
            ok = (d.view(np.uint64) == h.view(np.uint64)) | (np.isnan(d) & np.isnan(h))
            assert ok.all(), (xs[~ok][:3], ys[~ok][:3])
