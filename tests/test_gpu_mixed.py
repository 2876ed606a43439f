"""Mixed-precision form (FP32 inner PCG, FP64 refinement) against the FP64 oracle.

Tolerances (stated): FP32 matvec within 2e-6 of max|K x| (FP32 accumulation of 24-term rows over 8 elements);
solves to the same FP64 residual tolerance agree in compliance to 1e-8 relative and in u to 1e-6 of max|u|;
the SIMP loop agrees in compliance to 1e-6 relative per iteration (the accuracy the mixed form is specified to).
"""
import numpy as np
import pytest

from mycel_b200 import api
from mycel_b200 import workloads as W
from mycel_b200.model import StaticAnalysisOptions
from models import carved_model, tiny_test_model

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def exact_oracle(oracle):
    oracle.set_modes(0, threads=8)
    yield
    oracle.set_modes(0)


@pytest.mark.parametrize("variant", [1, 2, 3], ids=["dense", "tensor", "factored"])
@pytest.mark.parametrize("shape", [(1, 1, 1), (5, 3, 2), (33, 17, 9), (70, 9, 20), (16, 8, 3)])
def test_fp32_matvec_close_to_fp64(oracle, ctx, shape, variant):
    m = carved_model(*shape, seed=3, frac=0.15) if shape[0] > 2 else tiny_test_model(*shape)
    om, pr = oracle.Model(m), api.Problem(m, ctx)
    pr.set_matvec32(variant)
    assert pr.matvec32() == variant
    x = np.random.default_rng(2).uniform(-1, 1, m.total_dofs)
    y64 = om.apply_k(x)
    y32 = pr.apply_k(x, precision="mixed")
    assert np.abs(y32 - y64).max() <= 2e-6 * np.abs(y64).max()
    xp = x * (om.constrained() == 0)
    assert np.abs(pr.apply_k(xp, True, "mixed") - om.apply_a(xp)).max() <= 2e-6 * np.abs(y64).max()


def test_mixed_static_solve_matches_fp64(oracle, ctx):
    m = carved_model(24, 10, 8, seed=5, emin_ratio=1e-9)
    ref = oracle.static_run(m, 1e-10, 20000)
    r = api.StaticAnalysis.run(m, StaticAnalysisOptions(tolerance=1e-10, max_iterations=20000, precision="mixed"), ctx)
    assert r.solver_info.converged and r.solver_info.final_residual <= 1e-10
    assert abs(r.compliance - ref.compliance) <= 1e-8 * abs(ref.compliance)
    assert np.abs(r.u - ref.u).max() <= 1e-6 * np.abs(ref.u).max()
    assert np.array_equal(r.u[m.fixed_dofs], np.zeros(m.fixed_dofs.size))


@pytest.mark.parametrize("variant", [1, 2, 3], ids=["dense", "tensor", "factored"])
def test_mixed_pcg_each_matvec_variant(oracle, ctx, variant):
    m = carved_model(31, 12, 9, seed=8, emin_ratio=1e-9)
    om, pr = oracle.Model(m), api.Problem(m, ctx)
    pr.set_matvec32(variant)
    b = om.forces() * (om.constrained() == 0)
    ref, _ = om.pcg_solve(b, tol=1e-10, max_iter=20000)
    u, r = pr.pcg_solve(b, tol=1e-10, max_iterations=20000, precision="mixed")
    assert r.converged and r.final_residual <= 1e-10
    assert np.abs(u - ref).max() <= 1e-6 * np.abs(ref).max()
    assert pr.matvec32() == variant


def test_mixed_warm_start_and_zero_rhs(ctx):
    m = tiny_test_model()
    pr = api.Problem(m, ctx)
    b = pr.forces()
    u1, r1 = pr.pcg_solve(b, tol=1e-9, precision="mixed")
    u2, r2 = pr.pcg_solve(b, x0=u1, tol=1e-9, precision="mixed")
    assert r1.converged and r2.converged and r2.iterations <= 2
    u0, r0 = pr.pcg_solve(np.zeros(m.total_dofs), x0=np.ones(m.total_dofs), precision="mixed")
    assert r0.converged and not u0.any()


def test_mixed_simp_cantilever_within_1e6(oracle, ctx):
    m, o = W.simp_cantilever_40x20x10()
    o = o.replace(max_iterations=12)
    ref = oracle.topopt_run(m, o)
    res = api.TopologyOptimizer.run(m, o.replace(precision="mixed"), ctx=ctx)
    assert res.total_iterations == ref.n_iters
    for a, b in zip(res.snapshots, ref.records):
        assert abs(a.compliance - b["compliance"]) <= 1e-6 * abs(b["compliance"])
        assert a.solver_residual <= 1e-8
    assert np.abs(res.final_physical_density - ref.phys).max() <= 1e-5


def test_mixed_solve_finishes_in_fp64_when_inner_iterations_run_out(oracle, ctx):
    """An iteration budget the FP32 inner loop alone cannot meet: the solve is finished by the FP64 PCG from
    the refined solution, reports both counts, and matches the FP64 oracle to the solve tolerance."""
    m = carved_model(31, 12, 9, seed=8, emin_ratio=1e-9)
    om, pr = oracle.Model(m), api.Problem(m, ctx)
    b = om.forces() * (om.constrained() == 0)
    ref, _ = om.pcg_solve(b, tol=1e-8, max_iter=20000)
    _u0, r0 = pr.pcg_solve(b, tol=1e-8, max_iterations=20000, precision="mixed")
    assert r0.converged and r0.fallback_iterations == 0
    budget = int(r0.inner_iterations * 0.75)
    pr2 = api.Problem(m, ctx)  # a fresh problem: its first mixed solve runs the FP32 form
    u, r = pr2.pcg_solve(b, tol=1e-8, max_iterations=budget, precision="mixed")
    assert r.inner_iterations <= budget
    assert r.fallback_iterations > 0 and r.iterations == r.inner_iterations + r.fallback_iterations
    assert r.converged and r.final_residual <= 1e-8
    assert np.abs(u - ref).max() <= 1e-5 * np.abs(ref).max()


# ---- fast FP64 form (factorised operator, FP64 recurrences) ----
# Tolerances (stated): the factorised FP64 operator equals the Gauss KE product up to FP64 rounding, within
# 1e-12 of max|K x|; a solve to relative residual 1e-10 agrees with the FP64 oracle in u to 1e-7 of max|u| and
# needs no more than 1.2x the oracle's iterations (+10); SIMP compliance within 1e-7 per iteration.

@pytest.mark.parametrize("shape", [(1, 1, 1), (5, 3, 2), (33, 17, 9), (70, 9, 20)])
def test_fp64_factored_matvec_matches_oracle(oracle, ctx, shape):
    m = carved_model(*shape, seed=3, frac=0.15) if shape[0] > 2 else tiny_test_model(*shape)
    om, pr = oracle.Model(m), api.Problem(m, ctx)
    x = np.random.default_rng(2).uniform(-1, 1, m.total_dofs)
    y64 = om.apply_k(x)
    assert np.abs(pr.apply_k(x, precision="fp64f") - y64).max() <= 1e-12 * np.abs(y64).max()
    xp = x * (om.constrained() == 0)
    assert np.abs(pr.apply_k(xp, True, "fp64f") - om.apply_a(xp)).max() <= 1e-12 * np.abs(y64).max()


def test_fp64_factored_solve_matches_oracle(oracle, ctx):
    m = carved_model(31, 12, 9, seed=8, emin_ratio=1e-9)
    om, pr = oracle.Model(m), api.Problem(m, ctx)
    b = om.forces() * (om.constrained() == 0)
    ref, rref = om.pcg_solve(b, tol=1e-10, max_iter=20000)
    u, r = pr.pcg_solve(b, tol=1e-10, max_iterations=20000, precision="fp64f")
    assert r.converged and r.final_residual <= 1e-10 and r.fallback_iterations == 0
    assert r.iterations <= 1.2 * rref.iterations + 10
    assert np.abs(u - ref).max() <= 1e-7 * np.abs(ref).max()


def test_fp64_factored_simp_cantilever(oracle, ctx):
    m, o = W.simp_cantilever_40x20x10()
    o = o.replace(max_iterations=8)
    ref = oracle.topopt_run(m, o)
    res = api.TopologyOptimizer.run(m, o.replace(precision="fp64f"), ctx=ctx)
    assert res.total_iterations == ref.n_iters
    for a, b in zip(res.snapshots, ref.records):
        assert abs(a.compliance - b["compliance"]) <= 1e-7 * abs(b["compliance"])


def test_runwriter_frames_match_oracle(oracle, ctx):
    """Device-quantised frames of consecutive iterations equal RunWriter's bytes and FNV-1a checksums of the
    physical density snapshot (bit for bit), with the 72-byte header of the iteration."""
    import struct
    m, o = W.simp_cantilever_40x20x10()
    pr = api.Problem(m, ctx)
    sess = api.SimpSession(pr, o.replace(max_iterations=3))
    rolling = 2166136261
    for _ in range(3):
        rec = sess.step()
        slot = sess.frame_begin()
        phys = sess.read(u=False, densities=True)["physical"]
        q_ref, ck_ref = oracle.quantized_frame(phys)
        frame, header, ck = sess.frame_end(slot)
        assert np.array_equal(frame, q_ref) and ck == ck_ref
        magic, ver, nx, ny, nz, it = struct.unpack_from("<4s5i", header, 0)
        assert (magic, ver, nx, ny, nz, it) == (b"TOPO", 1, 40, 20, 10, rec.iteration)
        assert struct.unpack_from("<d", header, 24)[0] == rec.compliance
        assert struct.unpack_from("<I", header, 68)[0] == ck
        rolling = ((rolling ^ ck) * 16777619) & 0xFFFFFFFF
    assert rolling != 2166136261
    sess.close()
    pr.close()


def test_mixed_form_choice_is_per_problem_and_deterministic(oracle, ctx):
    """Second mixed solve of a problem probes the fast FP64 form; the choice after that rests on iteration
    counts, so two identical problems make the same choices and give the same bits."""
    m = carved_model(31, 12, 9, seed=8, emin_ratio=1e-9)
    runs = []
    for _ in range(2):
        pr = api.Problem(m, ctx)
        b = pr.forces()
        out = []
        for k in range(4):
            u, r = pr.pcg_solve(b, tol=1e-8, max_iterations=20000, precision="mixed")
            out.append((r.inner_iterations, r.fallback_iterations, u))
        runs.append(out)
        pr.close()
    assert runs[0][1][0] == 0 and runs[0][1][1] > 0  # the probe ran in fast FP64
    for a, b in zip(runs[0], runs[1]):
        assert a[0] == b[0] and a[1] == b[1] and np.array_equal(a[2], b[2])
