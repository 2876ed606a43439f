"""Pins of the CPU oracle against the reference's own known-answer tests and published numbers.

The reference (C#) cannot run here; these are the checks that make the oracle trustworthy:
Hex8ElementTests.cs:10-237 (KE), FemValidationTests.cs (V1, V3, V5, V9, V12, V13, V16, V17),
OptimizationTests.cs (T1-T7) and docs/VALIDATION.md:108-111 (V3 tip deflections, 4 decimals).
"""
import numpy as np
import pytest

from mycel_b200 import workloads as W
from mycel_b200.model import (ArgumentError, FeMaterial, FeModel, GridSpec, InvalidOperationError, LoadCase,
                              OptimizerOptions, SurfacePatch)
from models import bar_model, l_shape_domain, tiny_test_model, underconstrained_model

COORDS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)


# ---------------- Hex8 element (Hex8ElementTests.cs) ----------------
def test_ke_symmetric_and_rigid_modes(oracle):
    ke = oracle.create_ke(1.0, 0.3)
    assert ke.shape == (24, 24)
    assert np.abs(ke - ke.T).max() < 1e-12
    for axis in range(3):
        u = np.zeros(24)
        u[axis::3] = 1.0
        assert np.abs(ke @ u).max() < 1e-12
    th = 1e-3
    for rot in range(3):
        u = np.zeros((8, 3))
        c = COORDS - 0.5
        if rot == 0:
            u[:, 1], u[:, 2] = -th * c[:, 2], th * c[:, 1]
        elif rot == 1:
            u[:, 0], u[:, 2] = th * c[:, 2], -th * c[:, 0]
        else:
            u[:, 0], u[:, 1] = -th * c[:, 1], th * c[:, 0]
        assert np.abs(ke @ u.reshape(-1)).max() < 1e-12


def test_ke_patch_tests(oracle):
    nu, eps = 0.3, 0.001
    ke = oracle.create_ke(1.0, nu)
    u = np.zeros(24)
    for a in (1, 2, 5, 6):
        u[3 * a] = eps
    f = (ke @ u).reshape(8, 3)
    fac = 1.0 / ((1 + nu) * (1 - 2 * nu))
    sxx, syy = fac * (1 - nu) * eps / 4, fac * nu * eps / 4
    for a in range(8):
        assert abs(f[a, 0] - (sxx if COORDS[a, 0] else -sxx)) < 1e-12
        assert abs(f[a, 1] - (syy if COORDS[a, 1] else -syy)) < 1e-12
        assert abs(f[a, 2] - (syy if COORDS[a, 2] else -syy)) < 1e-12
    # pure shear u_x = gamma y
    u = np.zeros(24)
    for a in (2, 3, 6, 7):
        u[3 * a] = eps
    f = (ke @ u).reshape(8, 3)
    tau = eps / (2 * (1 + nu)) / 4
    for a in range(8):
        assert abs(f[a, 0] - (tau if COORDS[a, 1] else -tau)) < 1e-12
        assert abs(f[a, 1] - (tau if COORDS[a, 0] else -tau)) < 1e-12
        assert abs(f[a, 2]) < 1e-12


def test_ke_scaling_law(oracle):
    ke1 = oracle.create_ke(1.0, 0.28)
    for h in (0.5, 2.0, 3.5, 10.0):
        assert np.abs(oracle.create_ke(h, 0.28) - h * ke1).max() < 1e-12
    with pytest.raises(ArgumentError):
        oracle.create_ke(0.0, 0.3)


# ---------------- FEM validation (FemValidationTests.cs) ----------------
def test_v1_axial_bar(oracle):
    L, b, d, h, E, P = 100.0, 10.0, 10.0, 2.5, 3000.0, 1000.0
    model, tip = bar_model(L, b, d, h, E, 0.0)
    model.loads.append(LoadCase(tip, (P, 0, 0)))
    r = oracle.static_run(model, 1e-10, 5000)
    assert r.solver_info.converged
    ux = r.u[3 * tip.nodes]
    assert np.abs(ux - P * L / (b * d * E)).max() < 1e-6
    m = oracle.Model(model)
    vm = m.von_mises(r.u).reshape(model.grid.nz, model.grid.ny, model.grid.nx)
    assert np.abs(vm[:, :, 5:36] - P / (b * d)).max() < 1e-6


@pytest.mark.parametrize("nz,expected", [(1, 86.3730), (2, 116.7719), (4, 128.6479), (8, 132.1529)])
def test_v3_timoshenko_published_deflections(oracle, nz, expected):
    # docs/VALIDATION.md:108-111 — FE tip deflections printed to 4 decimals
    L, d, E, P = 100.0, 10.0, 3000.0, 1000.0
    h = d / nz
    model, tip = bar_model(L, d, d, h, E, 0.3)
    model.loads.append(LoadCase(tip, (0, 0, -P)))
    r = oracle.static_run(model, 1e-8, 10000)
    a = tip.node_area
    delta = (np.abs(r.u[3 * tip.nodes + 2]) * a).sum() / a.sum()
    assert round(delta, 4) == pytest.approx(expected, abs=1e-9)


def test_v5_energy_and_v9_scalar_reference(oracle):
    model, tip = bar_model(60.0, 10.0, 10.0, 2.5, 3000.0, 0.3)
    model.loads.append(LoadCase(tip, (500.0, 0, -500.0)))
    r = oracle.static_run(model, 1e-10, 5000)
    m = oracle.Model(model)
    ku = m.apply_k(r.u)
    assert abs(r.compliance - r.u @ ku) / abs(r.compliance) < 1e-8
    x = np.random.default_rng(42).uniform(-1, 1, model.total_dofs)
    y1, y2 = m.apply_k(x), m.apply_k_scalar_reference(x)
    assert (np.abs(y1 - y2) / np.maximum(1.0, np.abs(y2))).max() < 1e-12
    r2 = oracle.static_run(model, 1e-10, 5000)
    assert r2.solver_info.iterations == r.solver_info.iterations
    assert np.array_equal(r.u, r2.u) and np.array_equal(r.reactions, r2.reactions)


def test_v12_underconstrained_message(oracle):
    with pytest.raises(InvalidOperationError, match="(?i)sufficiently constrained"):
        oracle.static_run(underconstrained_model(), 1e-6, 500)


def test_preflight_fewer_than_six(oracle):
    g = GridSpec(2, 2, 2, 1.0)
    m = FeModel(g, np.ones(8), FeMaterial(1000.0, 0.3), [0, 1, 2],
                [LoadCase(SurfacePatch([26], [1.0]), (0, 0, -1))])
    with pytest.raises(InvalidOperationError, match="fewer than 6 unique fixed DOFs"):
        oracle.static_run(m)


def test_v13_warm_start_exact_zero_iterations(oracle):
    g = GridSpec(6, 2, 2, 1.0)
    fixed = FeModel.fix_dofs([g.node_index(0, j, k) for k in range(3) for j in range(3)])
    m = FeModel(g, np.ones(24), FeMaterial(1000.0, 0.3), fixed,
                [LoadCase(SurfacePatch([g.node_index(6, 1, 1)], [1.0]), (0, 0, -10.0))])
    cold = oracle.static_run(m, 1e-6)
    warm = oracle.static_run(m, 1e-6, warm_start=cold.u)
    assert cold.solver_info.iterations > 0 and warm.solver_info.iterations == 0
    assert warm.compliance == pytest.approx(cold.compliance, abs=1e-10)


def test_v16_unprojected_rhs(oracle):
    g = GridSpec(4, 2, 2, 1.0)
    fixed = FeModel.fix_dofs([g.node_index(0, j, k) for k in range(3) for j in range(3)])
    m = oracle.Model(FeModel(g, np.ones(16), FeMaterial(1000.0, 0.3), fixed))
    b = np.zeros(m.fe.total_dofs)
    b[3 * g.node_index(4, 1, 1) + 2] = -50.0
    b2 = b.copy()
    b2[fixed] = 12345.67
    u1, r1 = m.pcg_solve(b2, tol=1e-6)
    u2, r2 = m.pcg_solve(b, tol=1e-6)
    assert r1.converged and r2.converged
    assert np.all(u1[fixed] == 0.0)
    assert np.abs(u1 - u2).max() < 1e-10


def test_v17_bad_warm_start_length(oracle):
    g = GridSpec(2, 2, 2, 1.0)
    m = FeModel(g, np.ones(8), FeMaterial(1000.0, 0.3), FeModel.fix_dofs([0, 1]))
    with pytest.raises(ArgumentError):
        oracle.static_run(m, warm_start=np.zeros(m.total_dofs - 1))


def test_model_validation_errors():
    g = GridSpec(2, 2, 2, 1.0)
    with pytest.raises(ArgumentError):
        FeModel(g, np.ones(7), FeMaterial(1.0, 0.3), [])
    with pytest.raises(ArgumentError):
        FeModel(g, np.ones(8), FeMaterial(1.0, 0.3), [g.total_dofs])
    with pytest.raises(ArgumentError):
        GridSpec(0, 1, 1)


def test_force_conservation(oracle):
    # FeModelTests.cs:53 — forces sum to the total load within 1e-12 relative
    m = tiny_test_model()
    f = oracle.Model(m).forces().reshape(-1, 3).sum(0)
    assert np.allclose(f, [50.0, -30.0, -100.0], rtol=1e-12, atol=0)


# ---------------- SIMP (OptimizationTests.cs) ----------------
def test_t1_finite_difference_gradients(oracle):
    m = tiny_test_model()
    na = m.active_element_count
    rng = np.random.default_rng(12345)
    rho = 0.2 + 0.7 * rng.random(na)
    filt = oracle.Filter(m.grid, m.domain, m.active_elements, 1.8)
    rb = filt.apply(rho)
    m.element_density[m.active_elements] = rb
    base = oracle.static_run(m, 1e-12, 10000)
    om = oracle.Model(m)
    dcb = om.sensitivities(base.u, rb, 3.0)
    dc = filt.adjoint(dcb)
    hp = 1e-6
    for idx in rng.choice(na, 6, replace=False):
        for which in ("bar", "rho"):
            cs = []
            for sgn in (1, -1):
                if which == "bar":
                    d = rb.copy()
                    d[idx] += sgn * hp
                else:
                    r2 = rho.copy()
                    r2[idx] += sgn * hp
                    d = filt.apply(r2)
                m.element_density[m.active_elements] = d
                cs.append(oracle.static_run(m, 1e-12, 10000, warm_start=base.u).compliance)
            fd = (cs[0] - cs[1]) / (2 * hp)
            an = dcb[idx] if which == "bar" else dc[idx]
            assert abs(fd - an) / abs(an) < 1e-5
        m.element_density[m.active_elements] = rb
    s = filt.s
    for idx in range(0, na, 7):
        r2p, r2m = rho.copy(), rho.copy()
        r2p[idx] += hp
        r2m[idx] -= hp
        fd = (filt.apply(r2p).sum() - filt.apply(r2m).sum()) / (2 * hp)
        assert abs(fd - s[idx]) / s[idx] < 1e-5


def test_t2_filter_properties(oracle):
    g, dom = l_shape_domain()
    act = np.nonzero(dom)[0].astype(np.int32)
    f = oracle.Filter(g, dom, act, 2.5)
    assert np.abs(f.apply(np.full(act.size, 0.42)) - 0.42).max() < 1e-12
    s = f.s
    assert (s > 0).all() and abs(s.sum() - act.size) < 1e-10
    rng = np.random.default_rng(42)
    x, y = rng.random(act.size), rng.random(act.size)
    d1, d2 = f.apply(x) @ y, x @ f.adjoint(y)
    assert abs(d1 - d2) / abs(d1) < 1e-12


def test_t3_oc_fuzz(oracle):
    n = 200
    rng = np.random.default_rng(98765)
    s = 0.5 + rng.random(n)
    s *= n / s.sum()
    pas = np.zeros(n, np.uint8)
    pas[rng.integers(0, n, 20)] = 1
    rho = np.where(pas == 1, 1.0, 0.35)
    for _ in range(100):
        dc = -10.0 ** (-3.0 + 8.0 * rng.random(n))
        new, lam = oracle.oc_update(rho, dc, s, pas, 0.35, 0.2, 1e-3, 1.0)
        assert np.isfinite(lam) and lam > 0 and np.isfinite(new).all()
        assert (new >= 1e-3 - 1e-12).all() and (new <= 1 + 1e-12).all()
        assert (np.abs(new - rho) <= 0.2 + 1e-12).all()
        assert np.all(new[pas == 1] == 1.0)
        assert abs((s * new).sum() / n - 0.35) < 1e-6
        rho = new


def _cantilever_opts(**kw):
    return OptimizerOptions(volume_fraction=0.4, filter_radius_mm=2.0, penal=3.0, move_limit=0.2, max_iterations=25,
                            protect_boundary_hinges=False).replace(**kw)


def test_t4_t6_monotonic_and_sanity(oracle):
    m = W.cantilever(30, 10, 4)
    r = oracle.topopt_run(m, _cantilever_opts())
    c = [x["compliance"] for x in r.records]
    assert len(c) >= 15
    for i in range(5, len(c) - 1):
        assert c[i + 1] <= c[i] * 1.015
    mu = W.cantilever(30, 10, 4, element_density=np.full(1200, 0.4))
    assert r.records[-1]["compliance"] < oracle.static_run(mu, 1e-6).compliance
    assert abs(r.records[-1]["volume_fraction"] - 0.4) < 1e-3


def test_t5_bridge_mirror_symmetry(oracle):
    nx, ny, nz = 30, 1, 10
    g = GridSpec(nx, ny, nz, 1.0)
    fixed = FeModel.fix_dofs(sum(([g.node_index(0, j, 0), g.node_index(nx, j, 0)] for j in range(ny + 1)), []))
    ln = [g.node_index(nx // 2, j, 0) for j in range(ny + 1)]
    m = FeModel(g, np.ones(g.total_elements), FeMaterial(3000.0, 0.3, 1e-6), fixed,
                [LoadCase(SurfacePatch(ln, np.ones(len(ln))), (0, 0, -1000.0))])
    r = oracle.topopt_run(m, OptimizerOptions(volume_fraction=0.5, filter_radius_mm=2.0, max_iterations=20,
                                              protect_boundary_hinges=False))
    d = r.phys.reshape(nz, ny, nx)
    assert np.abs(d - d[:, :, ::-1]).max() < 1e-6


def test_t7_determinism_and_thread_independence(oracle):
    m = W.cantilever(20, 8, 4)
    o = _cantilever_opts(max_iterations=10)
    oracle.set_modes(0, threads=1)
    r1 = oracle.topopt_run(m, o)
    oracle.set_modes(0, threads=8)
    r2 = oracle.topopt_run(m, o)
    assert [x["compliance"] for x in r1.records] == [x["compliance"] for x in r2.records]
    assert np.array_equal(r1.phys, r2.phys) and np.array_equal(r1.u, r2.u)
    # restart from iteration 5 (design density + displacements) within 1e-4
    r5 = oracle.topopt_run(m, o.replace(max_iterations=5))
    rr = oracle.topopt_run(m, o.replace(start_iteration=6, initial_density=r5.design, warm_start_displacements=r5.u))
    assert abs(rr.records[-1]["compliance"] - r1.records[-1]["compliance"]) / r1.records[-1]["compliance"] < 1e-4


def test_passive_region_build(oracle):
    # PassiveRegionTests: Chebyshev shell of radius 1 around a node marks the <= 8 touching elements
    g = GridSpec(4, 4, 4, 1.0)
    out = oracle.passive_region(g, [g.node_index(2, 2, 2)], radius=1)
    assert out.sum() == 8
    out = oracle.passive_region(g, [g.node_index(0, 0, 0)], radius=1)
    assert out.sum() == 1 and out[0] == 1


# ---- RunWriter frames: FNV-1a 32-bit (published test vectors) and the 8-bit quantisation ----
def _frame_of_bytes(bs):
    # densities that quantise to the given byte values (v = b / 255 rounds back to b)
    return np.array([b / 255.0 for b in bs], dtype=np.float32)


def test_quantized_checksum_fnv1a_known_answers():
    from oracle import oracle as O
    assert O.quantized_frame(np.zeros(0, dtype=np.float32))[1] == 0x811C9DC5
    q, ck = O.quantized_frame(_frame_of_bytes(b"a"))
    assert list(q) == [97] and ck == 0xE40C292C
    q, ck = O.quantized_frame(_frame_of_bytes(b"foobar"))
    assert bytes(q) == b"foobar" and ck == 0xBF9CF968


def test_quantization_rounds_half_away_and_clamps():
    from oracle import oracle as O
    v = np.array([-0.5, 0.0, 1.0, 2.0, np.float32(0.5) / np.float32(255.0), 1.5 / 255.0, 0.5, 0.25],
                 dtype=np.float32)
    q, _ = O.quantized_frame(v)
    assert q[6] == 128  # 0.5 * 255 = 127.5 exactly: half away from zero
    expect = [0, 0, 255, 255]
    for x in v[4:]:
        c = np.float32(min(max(float(x), 0.0), 1.0)) * np.float32(255.0)
        f = np.floor(np.float64(c))
        expect.append(int(f + 1 if np.float64(c) - f >= 0.5 else f))
    assert list(q) == expect


def test_average_element_to_node_reference_case(oracle):
    """StaticAnalysisTests.AverageElementToNode_AveragesSharedElementsCorrectly: 2x2x1 grid, scalars 10..40,
    centre node (1,1,0) = 25, corner node (0,0,0) = 10."""
    from mycel_b200.model import FeMaterial, FeModel, GridSpec
    g = GridSpec(2, 2, 1, 1.0)
    m = FeModel(g, np.ones(4, dtype=np.uint8), FeMaterial(1000.0, 0.3), [0, 1, 2, 3, 4, 5])
    out = oracle.Model(m).average_element_to_node(np.array([10.0, 20.0, 30.0, 40.0]))
    assert abs(out[g.node_index(1, 1, 0)] - 25.0) < 1e-10
    assert abs(out[g.node_index(0, 0, 0)] - 10.0) < 1e-10


# Published PCG iteration counts of the reference's V10 scaling benchmark (docs/STEP3_BENCH.md:25-28), model
# of FemValidationTests.cs:633-726: cold solve to 1e-4 (rho = 1), warm solve to 1e-4 of the 2 % perturbed model
# (rho = 0.98) from the cold u, cold solve of the perturbed model, cold solve to 1e-6.
V10_PUBLISHED = {53_240: (436, 410, 436, 481), 98_415: (535, 503, 535, 591)}


def v10_counts(oracle, target):
    m0 = W.v10_cantilever(target)
    mp = W.v10_cantilever(target, 0.98)
    c4 = oracle.static_run(m0, 1e-4)
    w4 = oracle.static_run(mp, 1e-4, warm_start=c4.u)
    cp = oracle.static_run(mp, 1e-4)
    c6 = oracle.static_run(m0, 1e-6)
    return m0, (c4, w4, cp, c6)


def test_v10_published_pcg_counts_53k(oracle):
    # the whole PCG path (KE, forces, colour-ordered products, 8192-block reductions, stopping rule) reproduces
    # the reference's own published iteration counts
    oracle.set_modes(0, threads=8)
    m0, runs = v10_counts(oracle, 50_000)
    assert m0.total_elements == 53_240 and m0.total_dofs == 176_157
    assert tuple(r.solver_info.iterations for r in runs) == V10_PUBLISHED[53_240]


def test_lane_order_noise_floor(oracle):
    """The one detail of the reference that cannot be observed here, Vector256<double>.Sum's lane order, moves
    the 40x20x10 SIMP cantilever (30 iterations, reference defaults) by less than 1e-9 relative in compliance
    and 1e-7 relative in u: the bound on parity with the C# binary itself. Prints the spread table."""
    m, o = W.simp_cantilever_40x20x10()
    runs = {}
    for lane in (0, 1, 2):
        oracle.set_modes(lane, threads=8)
        runs[lane] = oracle.topopt_run(m, o)
    oracle.set_modes(0, threads=8)
    base = runs[0]
    for lane in (1, 2):
        r = runs[lane]
        c = max(abs(a["compliance"] - b["compliance"]) / abs(b["compliance"]) for a, b in zip(r.records, base.records))
        d = float(np.abs(r.phys - base.phys).max())
        u = float(np.abs(r.u - base.u).max() / np.abs(base.u).max())
        its = [a["solver_iterations"] - b["solver_iterations"] for a, b in zip(r.records, base.records)]
        print(f"lane mode {lane}: max rel compliance {c:.2g}, max abs rho_phys {d:.2g}, max rel u {u:.2g}, "
              f"PCG iteration differences {min(its)}..{max(its)}")
        assert c < 1e-9 and u < 1e-7
