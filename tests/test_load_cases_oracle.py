"""Separate load cases (multi-RHS over one stiffness, objective sum_k c_k) in the oracle.

The reference sums its load cases into one right-hand side (FeModel.AssembleForces, FeModel.cs:263-321) and has
no multi-load objective, so these semantics are pinned by the reference's own single-load pieces: each case's
solve equals StaticAnalysis.Run on the model holding that case alone, and the summed sensitivities are checked
against central finite differences of sum_k c_k (the T1 test of OptimizationTests.cs applied to the sum).
"""
import numpy as np

from mycel_b200 import workloads as W
from mycel_b200.model import FeModel, OptimizerOptions

from models import tiny_test_model


def _single(m, k, density=None):
    return FeModel(m.grid, m.domain, m.material, m.fixed_dofs, [m.loads[k]],
                   element_density=m.element_density if density is None else density, penal=m.penal)


def test_case_forces_sum_to_assembled_forces(oracle):
    m = tiny_test_model()
    om = oracle.Model(m)
    assert om.load_case_count() == 2
    f0, f1 = om.case_forces(0), om.case_forces(1)
    assert np.array_equal(f0, oracle.Model(_single(m, 0)).forces())
    assert np.array_equal(f1, oracle.Model(_single(m, 1)).forces())
    assert np.allclose(f0 + f1, om.forces(), rtol=0, atol=1e-15)


def test_multi_load_finite_difference_gradient(oracle):
    m = tiny_test_model()
    na = m.active_element_count
    rng = np.random.default_rng(2468)
    rb = 0.2 + 0.7 * rng.random(na)
    dens = m.element_density.copy()
    dens[m.active_elements] = rb
    singles = [_single(m, k, dens) for k in range(2)]
    base = [oracle.static_run(s, 1e-12, 10000) for s in singles]
    om = oracle.Model(singles[0])
    dcb = om.sensitivities(base[0].u, rb, 3.0) + om.sensitivities(base[1].u, rb, 3.0)
    hp = 1e-6
    for idx in rng.choice(na, 6, replace=False):
        cs = []
        for sgn in (1, -1):
            d = dens.copy()
            d[m.active_elements[idx]] += sgn * hp
            c = 0.0
            for k, s in enumerate(singles):
                s.element_density[:] = d
                c += oracle.static_run(s, 1e-12, 10000, warm_start=base[k].u).compliance
            cs.append(c)
        fd = (cs[0] - cs[1]) / (2 * hp)
        assert abs(fd - dcb[idx]) / abs(dcb[idx]) < 1e-5


def _opts(**kw):
    return OptimizerOptions(volume_fraction=0.4, filter_radius_mm=1.5, penal=3.0, max_iterations=6,
                            solver_tolerance_initial=1e-12, solver_tolerance_final=1e-12,
                            protect_boundary_hinges=False).replace(**kw)


def test_separate_cases_first_iteration_matches_single_load_solves(oracle):
    m = tiny_test_model()
    r = oracle.topopt_run(m, _opts(max_iterations=1, separate_load_cases=True))
    # iteration 1 runs on the filtered uniform design; the same design through the single-load models
    rs = oracle.topopt_run(m, _opts(max_iterations=1))
    dens = m.element_density.copy()
    dens[m.active_elements] = rs.rho_phys_active
    sol = [oracle.static_run(_single(m, k, dens), 1e-12, 10000) for k in range(2)]
    c = sol[0].compliance + sol[1].compliance
    assert abs(r.records[0]["compliance"] - c) / c < 1e-9
    assert np.abs(r.u - (sol[0].u + sol[1].u)).max() < 1e-9 * np.abs(r.u).max()
    md = max(np.sqrt((s.u.reshape(-1, 3) ** 2).sum(1)).max() for s in sol)
    assert abs(r.records[0]["max_displacement"] - md) / md < 1e-9


def test_separate_with_one_case_is_the_summed_run(oracle):
    m = W.cantilever(20, 8, 4)
    assert len(m.loads) == 1
    a = oracle.topopt_run(m, _opts(solver_tolerance_initial=1e-8, solver_tolerance_final=1e-8))
    b = oracle.topopt_run(m, _opts(solver_tolerance_initial=1e-8, solver_tolerance_final=1e-8,
                                   separate_load_cases=True))
    assert [x["compliance"] for x in a.records] == [x["compliance"] for x in b.records]
    assert np.array_equal(a.u, b.u) and np.array_equal(a.phys, b.phys)


def test_separate_cases_objective_decreases(oracle):
    m = tiny_test_model(nx=12, ny=6, nz=4)
    r = oracle.topopt_run(m, _opts(max_iterations=12, solver_tolerance_initial=1e-8, solver_tolerance_final=1e-8,
                                   separate_load_cases=True))
    c = [x["compliance"] for x in r.records]
    assert c[-1] < c[0]
    assert abs(r.records[-1]["volume_fraction"] - 0.4) < 1e-3


def test_separate_cases_with_an_empty_case(oracle):
    """A load case with no nodes and zero force (allowed by AssembleForces) adds a zero right-hand side: its
    solve returns u = 0 and the run equals the one without it."""
    from mycel_b200.model import LoadCase, SurfacePatch
    m = tiny_test_model()
    empty = LoadCase(SurfacePatch([], []), (0.0, 0.0, 0.0))
    m2 = FeModel(m.grid, m.domain, m.material, m.fixed_dofs, list(m.loads) + [empty])
    o = _opts(max_iterations=3, solver_tolerance_initial=1e-8, solver_tolerance_final=1e-8, separate_load_cases=True)
    a = oracle.topopt_run(m, o)
    b = oracle.topopt_run(m2, o)
    assert oracle.Model(m2).load_case_count() == 3
    assert not oracle.Model(m2).case_forces(2).any()
    assert [x["compliance"] for x in a.records] == [x["compliance"] for x in b.records]
    assert np.array_equal(a.phys, b.phys) and np.array_equal(a.u, b.u)
