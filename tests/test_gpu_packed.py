"""Packed solves (mycel_simp_step_many): the mixed multigrid SIMP iterations of several problems side by side,
every kernel of their FP32 outer iterations one launch for all of them (per-problem tables split the CTAs).

The reference runs one optimisation at a time (OptimizationCoordinator.cs:229, serialised by FemWorkTeam.cs:109);
its per-problem semantics are those of TopologyOptimizer.Run (TopologyOptimizer.cs:16-407). The packed form
must change nothing per problem: each problem's compliance, solver iteration counts, displacements and
densities are compared with its own session stepped alone, bit for bit (tolerance 0).
"""
import numpy as np
import pytest

from mycel_b200 import api
from mycel_b200 import workloads as W
from mycel_b200.model import OptimizerOptions

pytestmark = pytest.mark.gpu

ITERS = 3


def _jobs():
    """Grids of different multigrid depths (so the problems' levels differ in number and size), a bridge, a grid
    too small for separate coarse levels, and two problems whose load cases are kept apart (solved together
    within the pack)."""
    base = OptimizerOptions(volume_fraction=0.3, filter_radius_mm=1.5, max_iterations=ITERS, precision="mixed-mg",
                            solver_tolerance_initial=1e-6, solver_tolerance_final=1e-6, solver_max_iterations=20000)
    jobs = [
        (W.cantilever(24, 12, 8, e0=1.0, emin_ratio=1e-9, force=-1.0), base),
        (W.cantilever(60, 30, 16, e0=1.0, emin_ratio=1e-9, force=-1.0), base.replace(volume_fraction=0.2)),
        (W.bridge(48, 24, 24, support=4, load_patch=8), base.replace(volume_fraction=0.15, filter_radius_mm=2.5)),
        (W.cantilever(9, 5, 3, e0=1.0, emin_ratio=1e-9, force=-1.0), base),
    ]
    for bp in W.batched_instances(count=16, seed=7, scale=0.35):
        if len(bp.load_cases) >= 3:
            jobs.append((bp.model, bp.options.replace(max_iterations=ITERS, precision="mixed-mg",
                                                      separate_load_cases=True)))
        if len(jobs) == 6:
            break
    assert len(jobs) == 6
    return jobs


def _session(ctx, m, o):
    p = api.Problem(m, ctx)
    p.set_matvec32(3)  # the factorised matvec, which the packed form runs (the autotuner may pick another alone)
    return p, api.SimpSession(p, o)


def _alone(ctx, m, o, iters):
    p, s = _session(ctx, m, o)
    try:
        recs = [s.step() for _ in range(iters)]
        return recs, s.read()
    finally:
        s.close()
        p.close()


def _packed(ctx, jobs, iters):
    made = [_session(ctx, m, o) for m, o in jobs]
    try:
        sess = [s for _, s in made]
        recs = [[] for _ in sess]
        for _ in range(iters):
            for k, r in enumerate(api.SimpSession.step_many(sess)):
                recs[k].append(r)
        return recs, [s.read() for s in sess]
    finally:
        for p, s in made:
            s.close()
            p.close()


def _same(ra, da, rp, dp):
    assert len(ra) == len(rp)
    for a, b in zip(ra, rp):
        assert a.compliance == b.compliance
        assert a.solver_iterations == b.solver_iterations
        assert a.volume_fraction == b.volume_fraction
        assert a.max_change == b.max_change
    assert np.array_equal(da["u"], dp["u"])
    assert np.array_equal(da["physical"], dp["physical"])
    assert np.array_equal(da["design"], dp["design"])


def test_packed_iterations_equal_each_problem_alone(ctx):
    jobs = _jobs()
    alone = [_alone(ctx, m, o, ITERS) for m, o in jobs]
    before = ctx.packed_count
    rp, dp = _packed(ctx, jobs, ITERS)
    rhs = sum(len(m.loads) if o.separate_load_cases and len(m.loads) > 1 else 1 for m, o in jobs)
    assert ctx.packed_count - before == ITERS * rhs, "every solve ran through the packed launches"
    for k, (ra, da) in enumerate(alone):
        _same(ra, da, rp[k], dp[k])


def test_packed_twice_in_a_row_and_in_another_order(ctx):
    """A second batch (reversed order: new tables) gives the same bits again."""
    jobs = _jobs()[:4]
    r1, d1 = _packed(ctx, jobs, 2)
    r2, d2 = _packed(ctx, jobs[::-1], 2)
    n = len(jobs)
    for k in range(n):
        _same(r1[k], d1[k], r2[n - 1 - k], d2[n - 1 - k])


def test_other_forms_in_one_batch(ctx):
    """Sessions of other forms in the same batch are stepped alone inside the call; each equals its run alone."""
    jobs = _jobs()[:3]
    jobs[1] = (jobs[1][0], jobs[1][1].replace(precision="fp64", solver_tolerance_initial=1e-8,
                                              solver_tolerance_final=1e-8))
    alone = [_alone(ctx, m, o, 2) for m, o in jobs]
    rp, dp = _packed(ctx, jobs, 2)
    for k, (ra, da) in enumerate(alone):
        _same(ra, da, rp[k], dp[k])


def test_run_many_matches_run(ctx):
    m, o = _jobs()[0]
    o = o.replace(max_iterations=4)
    res = api.TopologyOptimizer.run_many([m, W.cantilever(30, 10, 6, e0=1.0, emin_ratio=1e-9, force=-1.0)], o,
                                         ctx=ctx)
    one = api.TopologyOptimizer.run(m, o, ctx=ctx)
    assert res[0].total_iterations == one.total_iterations == 4
    assert [s.compliance for s in res[0].snapshots] == [s.compliance for s in one.snapshots]
    assert np.array_equal(res[0].final_physical_density, one.final_physical_density)


def test_batch_arguments(ctx):
    m, o = _jobs()[0]
    p, s = _session(ctx, m, o)
    other = api.Context(0)
    try:
        q, t = _session(other, m, o)
        try:
            with pytest.raises(Exception, match="share one context"):
                api.SimpSession.step_many([s, t])
        finally:
            t.close()
            q.close()
        s2 = api.SimpSession(p, o)
        try:
            with pytest.raises(Exception, match="its own problem"):
                api.SimpSession.step_many([s, s2])
        finally:
            s2.close()
    finally:
        s.close()
        p.close()
        other.close()


def test_run_many_each_problem_as_alone(ctx):
    """Whole runs side by side (mycel_simp_run_many): each problem goes on to its next SIMP iteration as soon as
    its own solve ends; runs of different lengths end at different times. Each equals its run alone."""
    jobs = [(m, o.replace(max_iterations=2 + k % 3)) for k, (m, o) in enumerate(_jobs())]
    alone = [_alone(ctx, m, o, o.max_iterations) for m, o in jobs]
    made = [_session(ctx, m, o) for m, o in jobs]
    try:
        before = ctx.packed_count
        out = api.SimpSession.run_many([s for _, s in made])
        reads = [s.read() for _, s in made]
        rhs = sum((len(m.loads) if o.separate_load_cases and len(m.loads) > 1 else 1) * o.max_iterations
                  for m, o in jobs)
        assert ctx.packed_count - before == rhs, "every solve ran in the packed plan"
    finally:
        for p, s in made:
            s.close()
            p.close()
    for k, (ra, da) in enumerate(alone):
        _same(ra, da, out[k], reads[k])


def test_run_many_with_a_session_of_another_form(ctx):
    """A session the packed form cannot take (FP64 here) is stepped alone inside the run; all equal their runs
    alone."""
    jobs = _jobs()[:3]
    jobs[1] = (jobs[1][0], jobs[1][1].replace(precision="fp64", solver_tolerance_initial=1e-8,
                                              solver_tolerance_final=1e-8, max_iterations=2))
    alone = [_alone(ctx, m, o, o.max_iterations) for m, o in jobs]
    made = [_session(ctx, m, o) for m, o in jobs]
    try:
        out = api.SimpSession.run_many([s for _, s in made])
        reads = [s.read() for _, s in made]
    finally:
        for p, s in made:
            s.close()
            p.close()
    for k, (ra, da) in enumerate(alone):
        _same(ra, da, out[k], reads[k])


def test_read_into_caller_buffers(ctx):
    """SimpSession.read(out=...) fills the caller's (pinned or plain) arrays with what read() returns."""
    m, o = _jobs()[3]
    p, s = _session(ctx, m, o)
    try:
        s.step()
        ref = s.read(u=True, densities=True)
        out = {"u": np.empty(m.total_dofs), "physical": np.empty(m.total_elements, dtype=np.float32),
               "design": np.empty(m.total_elements, dtype=np.float32)}
        got = s.read(u=True, densities=True, out=out)
        for k in ("u", "physical", "design"):
            assert got[k] is out[k] and np.array_equal(got[k], ref[k])
        with pytest.raises(Exception, match="contiguous"):
            s.read(u=True, densities=False, out={"u": np.empty(3)})
    finally:
        s.close()
        p.close()


def test_run_many_cancelled_then_stepped_alone(ctx):
    """A cancelled packed run (CancellationToken, TopologyOptimizer.cs:169-172) returns without error and without
    records, and leaves the sessions to step on by themselves. Their next iteration is the first one again (the
    multigrid damping estimate may start warm, so its compliance is compared within 1e-5 relative: both solves
    meet the 1e-6 residual tolerance)."""
    jobs = _jobs()[:2]
    fresh = [_alone(ctx, m, o, 1) for m, o in jobs]
    made = [_session(ctx, m, o) for m, o in jobs]
    try:
        ctl = api.IterationController()
        ctl.stop()
        out = api.SimpSession.run_many([s for _, s in made], controller=ctl)
        assert all(len(r) == 0 for r in out)
        for k, (_, s) in enumerate(made):
            assert not s.done
            r = s.step()
            assert r.iteration == fresh[k][0][0].iteration
            assert abs(r.compliance - fresh[k][0][0].compliance) <= 1e-5 * abs(fresh[k][0][0].compliance)
    finally:
        for p, s in made:
            s.close()
            p.close()


def test_staged_level_product_equals_the_gather(ctx):
    """Coarse levels of more than 64k nodes: alone, their products run with the stencil staged by TMA
    (k_mg_apply_nodes_tma); packed, by the thread-per-node gather (k_mg_apply_nodes_pk). The two must give the
    same bits: an even bridge and an odd-sized cantilever (level 1: 81x41x21 and 82x42x22 nodes)."""
    o = OptimizerOptions(volume_fraction=0.3, filter_radius_mm=1.5, max_iterations=2, precision="mixed-mg",
                         solver_tolerance_initial=1e-6, solver_tolerance_final=1e-6, solver_max_iterations=20000)
    jobs = [(W.bridge(160, 80, 40, support=6, load_patch=10), o),
            (W.cantilever(161, 81, 41, e0=1.0, emin_ratio=1e-9, force=-1.0), o.replace(volume_fraction=0.2))]
    alone = [_alone(ctx, m, jo, 2) for m, jo in jobs]
    rp, dp = _packed(ctx, jobs, 2)
    for k, (ra, da) in enumerate(alone):
        _same(ra, da, rp[k], dp[k])
