"""Load cases kept apart (multi-RHS PCG over one stiffness, objective sum_k c_k) on the GPU, against the oracle.

The reference sums its load cases (FeModel.AssembleForces, FeModel.cs:263-321); each case's solve is pinned by
the oracle's StaticAnalysis of the model holding that case alone, and the multi-load SIMP loop by the oracle's
run of the same semantics (its sensitivities pinned by finite differences in test_load_cases_oracle.py).
"""
import numpy as np
import pytest

from mycel_b200 import api
from mycel_b200 import workloads as W
from mycel_b200.model import FeModel, OptimizerOptions, StaticAnalysisOptions

from models import tiny_test_model

pytestmark = pytest.mark.gpu


@pytest.fixture
def oracle_cr(oracle):
    """The reference-faithful oracle (the C library's pow, .NET 8+ lane order), as the device computes."""
    oracle.set_modes(0)
    yield oracle
    oracle.set_modes(0)


def _single(m, k):
    return FeModel(m.grid, m.domain, m.material, m.fixed_dofs, [m.loads[k]], element_density=m.element_density,
                   penal=m.penal)


def _multi_case_models():
    out = [tiny_test_model(nx=10, ny=5, nz=4)]
    for bp in W.batched_instances(count=12, seed=7, scale=0.25):
        if len(bp.load_cases) >= 3:
            out.append(bp.model)
        if len(out) == 3:
            break
    assert len(out) == 3
    return out


def test_case_forces_match_oracle(oracle, ctx):
    m = _multi_case_models()[1]
    prob = api.Problem(m, ctx)
    try:
        om = oracle.Model(m)
        assert prob.load_case_count() == om.load_case_count() == len(m.loads)
        for k in range(len(m.loads)):
            assert np.array_equal(prob.case_forces(k), om.case_forces(k))
    finally:
        prob.close()


@pytest.mark.parametrize("which", [0, 1, 2])
def test_static_cases_fp64(oracle_cr, ctx, which):
    """Case k: the same bits as the library's static solve of the model holding case k alone and as the
    oracle's StaticAnalysis of that model."""
    oracle = oracle_cr
    m = _multi_case_models()[which]
    rng = np.random.default_rng(which)
    m.element_density[:] = rng.uniform(0.1, 1.0, m.total_elements)
    opt = StaticAnalysisOptions(tolerance=1e-8, max_iterations=20000)
    got = api.StaticAnalysis.run_cases(m, opt, ctx=ctx)
    assert len(got) == len(m.loads)
    for k, g in enumerate(got):
        one = api.StaticAnalysis.run(_single(m, k), opt, ctx=ctx, reactions=False, von_mises=False)
        assert g.solver_info.iterations == one.solver_info.iterations
        assert np.array_equal(g.u, one.u)
        assert g.compliance == one.compliance and g.max_displacement == one.max_displacement
        ref = oracle.static_run(_single(m, k), 1e-8, 20000)
        assert g.solver_info.iterations == ref.solver_info.iterations
        assert np.array_equal(g.u, ref.u)
        assert g.compliance == ref.compliance and g.max_displacement == ref.max_displacement


@pytest.mark.parametrize("precision", ["mixed", "mg", "mixed-mg"])
def test_static_cases_refined_forms(oracle, ctx, precision):
    m = _multi_case_models()[1]
    rng = np.random.default_rng(5)
    m.element_density[:] = rng.uniform(0.1, 1.0, m.total_elements)
    got = api.StaticAnalysis.run_cases(m, StaticAnalysisOptions(tolerance=1e-10, max_iterations=20000,
                                                                precision=precision), ctx=ctx)
    for k, g in enumerate(got):
        ref = oracle.static_run(_single(m, k), 1e-12, 40000)
        assert g.solver_info.converged
        assert abs(g.compliance - ref.compliance) <= 1e-8 * abs(ref.compliance)
        assert np.abs(g.u - ref.u).max() <= 1e-7 * np.abs(ref.u).max()


def _opts(**kw):
    return OptimizerOptions(volume_fraction=0.3, filter_radius_mm=1.5, max_iterations=5, protect_boundary_hinges=False,
                            solver_tolerance_initial=1e-8, solver_tolerance_final=1e-8,
                            solver_max_iterations=20000, separate_load_cases=True).replace(**kw)


@pytest.mark.parametrize("which", [0, 1])
def test_simp_separate_cases_fp64_parity(oracle_cr, ctx, which):
    oracle = oracle_cr
    m = _multi_case_models()[which]
    o = _opts()
    ref = oracle.topopt_run(m, o)
    res = api.TopologyOptimizer.run(m, o, ctx=ctx)
    assert res.total_iterations == ref.n_iters
    for a, b in zip(res.snapshots, ref.records):
        assert a.solver_iterations == b["solver_iterations"]
        assert a.compliance == b["compliance"]
        assert a.max_change == b["max_change"]
        assert a.max_displacement == b["max_displacement"]
    assert np.array_equal(res.final_displacements, ref.u)
    assert np.array_equal(res.final_physical_density, ref.phys)
    assert np.array_equal(res.final_design_density, ref.design)


def test_simp_separate_cases_differ_from_summed(ctx):
    m = _multi_case_models()[0]
    a = api.TopologyOptimizer.run(m, _opts(max_iterations=2, separate_load_cases=False), ctx=ctx)
    b = api.TopologyOptimizer.run(m, _opts(max_iterations=2), ctx=ctx)
    assert a.snapshots[0].compliance != b.snapshots[0].compliance


def test_simp_separate_one_case_equals_summed(ctx):
    m = W.cantilever(16, 8, 4)
    a = api.TopologyOptimizer.run(m, _opts(separate_load_cases=False), ctx=ctx)
    b = api.TopologyOptimizer.run(m, _opts(), ctx=ctx)
    assert [s.compliance for s in a.snapshots] == [s.compliance for s in b.snapshots]
    assert np.array_equal(a.final_displacements, b.final_displacements)


@pytest.mark.parametrize("precision", ["mixed", "mixed-mg"])
def test_simp_separate_cases_mixed_within_tolerance(ctx, precision):
    m = _multi_case_models()[1]
    ref = api.TopologyOptimizer.run(m, _opts(), ctx=ctx)
    res = api.TopologyOptimizer.run(m, _opts(precision=precision), ctx=ctx)
    for a, b in zip(res.snapshots, ref.snapshots):
        assert abs(a.compliance - b.compliance) <= 1e-6 * abs(b.compliance)
    assert np.abs(res.final_design_density - ref.final_design_density).max() <= 1e-4


def test_simp_separate_cases_with_an_empty_case(oracle_cr, ctx):
    """A load case without nodes and force adds a zero right-hand side (the solvers' zero-RHS branch): the run
    equals the oracle's and the run without that case."""
    from mycel_b200.model import LoadCase, SurfacePatch
    m = _multi_case_models()[0]
    m2 = FeModel(m.grid, m.domain, m.material, m.fixed_dofs,
                 list(m.loads) + [LoadCase(SurfacePatch([], []), (0.0, 0.0, 0.0))])
    o = _opts(max_iterations=3)
    ref = oracle_cr.topopt_run(m2, o)
    for prec in ("fp64", "mixed-mg"):
        a = api.TopologyOptimizer.run(m, o.replace(precision=prec), ctx=ctx)
        b = api.TopologyOptimizer.run(m2, o.replace(precision=prec), ctx=ctx)
        assert [s.compliance for s in a.snapshots] == [s.compliance for s in b.snapshots]
        if prec == "fp64":
            assert [s.compliance for s in b.snapshots] == [r["compliance"] for r in ref.records]
            assert np.array_equal(b.final_physical_density, ref.phys)


@pytest.mark.parametrize("which", [0, 1, 2])
def test_static_cases_solved_together_equal_each_alone(ctx, which):
    """Mixed multigrid form: the cases of one stiffness are solved together (their outer iterations side by side,
    one V-cycle whose coarse levels advance every case per stencil read); each case gets the iterations and the
    bits of its solve alone."""
    m = _multi_case_models()[which]
    rng = np.random.default_rng(10 + which)
    m.element_density[:] = rng.uniform(0.1, 1.0, m.total_elements)
    opt = StaticAnalysisOptions(tolerance=1e-8, max_iterations=20000, precision="mixed-mg")
    got = api.StaticAnalysis.run_cases(m, opt, ctx=ctx)
    assert len(got) == len(m.loads) >= 2
    for k, g in enumerate(got):
        one = api.StaticAnalysis.run(_single(m, k), opt, ctx=ctx, reactions=False, von_mises=False)
        assert g.solver_info.converged and one.solver_info.converged
        assert g.solver_info.iterations == one.solver_info.iterations
        assert np.array_equal(g.u, one.u)
        assert g.compliance == one.compliance


def test_simp_cases_together_equal_one_after_another(ctx, monkeypatch):
    """The SIMP loop with load cases apart in the mixed multigrid form: solving the cases together gives the
    same iterates as solving them one after another (MYCEL_CASES_TOGETHER=0)."""
    m = _multi_case_models()[1]
    o = _opts(precision="mixed-mg", max_iterations=4)
    together = api.TopologyOptimizer.run(m, o, ctx=ctx)
    monkeypatch.setenv("MYCEL_CASES_TOGETHER", "0")
    apart = api.TopologyOptimizer.run(m, o, ctx=ctx)
    monkeypatch.delenv("MYCEL_CASES_TOGETHER")
    assert [s.compliance for s in together.snapshots] == [s.compliance for s in apart.snapshots]
    assert [s.solver_iterations for s in together.snapshots] == [s.solver_iterations for s in apart.snapshots]
    assert np.array_equal(together.final_displacements, apart.final_displacements)
    assert np.array_equal(together.final_design_density, apart.final_design_density)
