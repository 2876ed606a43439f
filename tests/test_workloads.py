"""The seeded synthetic workloads stand in for the benchmark configurations: their shapes, ranges and counts are
checked here (CPU only), so a change to a generator cannot silently change what is measured."""
import numpy as np

from mycel_b200 import workloads as W


def test_cantilever_40x20x10():
    m, o = W.simp_cantilever_40x20x10()
    g = m.grid
    assert (g.nx, g.ny, g.nz) == (40, 20, 10) and m.total_elements == 8000
    assert m.material.e0 == 1.0 and m.material.nu == 0.3 and m.material.emin_ratio == 1e-9
    assert o.volume_fraction == 0.3 and o.filter_radius_mm == 1.5 and o.penal == 3.0 and o.move_limit == 0.2
    assert o.max_iterations == 30 and o.solver_tolerance_initial == o.solver_tolerance_final == 1e-8
    assert o.solver_max_iterations == 2000
    # all DOFs of the x = 0 nodes fixed; total load -1 in z on the edge x = 40, z = 0
    assert m.fixed_dofs.size == 3 * 21 * 11
    (lc,) = m.loads
    assert lc.total_force == (0.0, 0.0, -1.0) and lc.patch.node_count == 21


def test_bridge_192x96x96():
    m, o = W.bridge_192x96x96()
    g = m.grid
    assert (g.nx, g.ny, g.nz) == (192, 96, 96) and m.total_elements == 1_769_472
    assert m.total_dofs == 3 * 193 * 97 * 97
    assert o.volume_fraction == 0.15 and o.filter_radius_mm == 2.5 and o.penal == 3.0 and o.max_iterations == 50
    # four 8 x 8 corner supports, fully fixed; one load of total 1 over a 16 x 16 top patch
    assert m.fixed_dofs.size == 4 * 8 * 8 * 3
    (lc,) = m.loads
    assert abs(np.linalg.norm(lc.total_force) - 1.0) < 1e-12 and lc.patch.node_count == 16 * 16


def test_sphere_carved_box():
    m = W.sphere_carved_box()
    g = m.grid
    assert (g.nx, g.ny, g.nz) == (96, 48, 24)
    assert abs(m.active_element_count - 98_400) / 98_400 < 0.01
    d = m.element_density[m.active_elements]
    assert d.min() >= 0.1 and d.max() <= 1.0


def test_batched_instances_match_their_configuration():
    probs = W.batched_instances()
    assert len(probs) == 48
    for bp in probs:
        g = bp.model.grid
        assert 24 <= g.nx <= 128 and g.ny == g.nx // 2 and 8 <= g.nz <= 64
        assert 1 <= len(bp.load_cases) <= 6 and bp.model.loads == bp.load_cases
        for lc in bp.load_cases:
            assert abs(np.linalg.norm(lc.total_force) - 1.0) < 1e-6
            assert lc.patch.node_count <= 16
        assert 0.1 <= bp.options.volume_fraction <= 0.4 and 1.2 <= bp.options.filter_radius_mm <= 3.0
    # the same seed gives the same problems
    again = W.batched_instances()
    assert [(p.model.grid.nx, p.model.grid.nz, len(p.load_cases)) for p in probs] == \
           [(p.model.grid.nx, p.model.grid.nz, len(p.load_cases)) for p in again]


def test_job_stream_matches_its_configuration():
    jobs = W.job_stream()
    assert len(jobs) == 500
    t = np.array([j[0] for j in jobs])
    assert np.all(np.diff(t) > 0)
    rate = len(jobs) / t[-1]
    assert 16.0 < rate < 24.0  # Poisson(20/s)
    it = np.array([j[4] for j in jobs])
    assert it.min() >= 20 and it.max() <= 60
    ne = np.array([j[1] * j[2] * j[3] for j in jobs])
    assert ne.min() >= 4_000 and ne.max() <= 1_300_000
