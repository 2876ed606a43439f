"""Serving loop (mycel_server): jobs run concurrently give the same results as alone; admission respects the
HBM budget; the admission estimate bounds the memory a job really holds; latency statistics are reported.

Tolerances (stated): FP64 jobs are bit-identical alone and in the mix (every reduction has a fixed order and
each job's kernels see only its own data); mixed jobs are too, because the FP32 matvec variant is chosen once
per grid for the whole process; the test still states 1e-12 relative on compliance for the mixed form.
"""
import numpy as np
import pytest

from mycel_b200 import api
from mycel_b200 import workloads as W
from mycel_b200.model import ArgumentError, OutOfMemoryError

pytestmark = pytest.mark.gpu


def _jobs(precision, n=5, iters=4):
    shapes = [(24, 12, 8), (32, 16, 8), (20, 10, 10), (28, 14, 6), (36, 12, 8), (16, 8, 8)]
    return [W.served_job(nx, ny, nz, iters, seed=100 + i, precision=precision)
            for i, (nx, ny, nz) in enumerate(shapes[:n])]


@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed-mg"])
def test_results_same_alone_and_in_mix(ctx, precision):
    jobs = _jobs(precision)
    alone = [api.TopologyOptimizer.run(m, o, ctx=ctx) for m, o in jobs]
    with api.Server(slots=3, hbm_budget_bytes=8 * 10**9) as srv:
        ids = [srv.submit(m, o, keep_u=True) for m, o in jobs]
        srv.wait()
        for jid, ref in zip(ids, alone):
            r = srv.result(jid, u=True)
            assert r["info"]["state"] == "done", r["info"]["message"]
            assert len(r["history"]) == ref.total_iterations
            for a, b in zip(r["history"], ref.snapshots):
                if precision == "fp64":
                    assert a.compliance == b.compliance
                else:
                    assert abs(a.compliance - b.compliance) <= 1e-12 * abs(b.compliance)
            if precision == "fp64":
                assert np.array_equal(r["physical"], ref.final_physical_density)
                assert np.array_equal(r["u"], ref.final_displacements)
            else:
                assert np.abs(r["physical"] - ref.final_physical_density).max() <= 1e-6
        st = srv.stats()
        assert st["completed"] == len(jobs) and st["failed"] == 0
        assert 0 < st["p50_latency_s"] <= st["p99_latency_s"] <= st["max_latency_s"]


def test_admission_respects_budget_and_rejects_oversize():
    jobs = _jobs("mixed", n=4, iters=2)
    sizes = [api.Server.device_bytes(m, o) for m, o in jobs]
    budget = int(max(sizes) * 1.5)  # room for one job at a time (and sometimes two small ones)
    big_m, big_o = W.served_job(64, 32, 32, 2, seed=9)
    with api.Server(slots=4, hbm_budget_bytes=budget) as srv:
        ids = [srv.submit(m, o) for m, o in jobs]
        big = srv.submit(big_m, big_o) if api.Server.device_bytes(big_m, big_o) > budget else None
        srv.wait()
        st = srv.stats()
        assert st["peak_admitted_bytes"] <= budget
        assert st["completed"] == len(jobs)
        for jid in ids:
            assert srv.info(jid)["state"] == "done"
        if big is not None:
            info = srv.info(big)
            assert info["state"] == "failed" and "budget" in info["message"]
            with pytest.raises(OutOfMemoryError):
                srv.result(big)


@pytest.mark.parametrize("precision", ["fp64", "mixed", "fp64f", "mg", "mixed-mg"])
def test_admission_estimate_bounds_job_memory(ctx, precision):
    m, o = W.served_job(30, 14, 10, 2, seed=5, precision=precision)
    est = api.Server.device_bytes(m, o)
    pr = api.Problem(m, ctx)
    sess = api.SimpSession(pr, o)
    sess.step()  # the first solve allocates the PCG (and mixed) workspaces
    held = pr.info()["device_bytes"]
    sess.close()
    pr.close()
    # the estimate also holds the fast FP64 workspace that a mixed solve allocates only if it escalates
    g = m.grid
    fast64 = 7 * (8 * ((3 * (g.nx + 1) + 1) // 2 * 2) * (g.ny + 1) * (g.nz + 1) + 64) if precision == "mixed" else 0
    assert held <= est <= 1.25 * held + fast64


def test_unknown_job_is_an_argument_error():
    with api.Server(slots=1, hbm_budget_bytes=10**9) as srv:
        with pytest.raises(ArgumentError):
            srv.info(12345)


@pytest.mark.parametrize("precision", ["fp64", "mixed-mg"])
def test_separate_load_cases_served(ctx, precision):
    """Jobs whose load cases are kept apart: same results alone and in the mix, estimate bounds their memory."""
    jobs = [(m, o.replace(separate_load_cases=True)) for m, o in _jobs(precision, n=4, iters=3)]
    assert sum(len(m.loads) > 1 for m, _ in jobs) >= 3
    alone = [api.TopologyOptimizer.run(m, o, ctx=ctx) for m, o in jobs]
    with api.Server(slots=3, hbm_budget_bytes=8 * 10**9) as srv:
        ids = [srv.submit(m, o) for m, o in jobs]
        srv.wait()
        for jid, ref in zip(ids, alone):
            r = srv.result(jid)
            assert r["info"]["state"] == "done", r["info"]["message"]
            for a, b in zip(r["history"], ref.snapshots):
                assert abs(a.compliance - b.compliance) <= (0.0 if precision == "fp64" else 1e-12) * abs(b.compliance)
    m, o = W.served_job(30, 14, 10, 2, seed=2, precision=precision)
    o = o.replace(separate_load_cases=True)
    assert len(m.loads) == 3
    est = api.Server.device_bytes(m, o)
    pr = api.Problem(m, ctx)
    sess = api.SimpSession(pr, o)
    sess.step()
    held = pr.info()["device_bytes"]
    sess.close()
    pr.close()
    assert held <= est <= 1.25 * held


def test_six_slots_started_together(ctx):
    """Six jobs admitted at once into six slots: their contexts' first OC launches overlap on the device; every
    job's results are still bit-identical to the job run alone (plain method)."""
    shapes = [(24, 12, 8), (32, 16, 8), (20, 10, 10), (28, 14, 6), (36, 12, 8), (16, 8, 8)]
    jobs = [W.served_job(nx, ny, nz, 3, seed=300 + i, precision="fp64") for i, (nx, ny, nz) in enumerate(shapes)]
    alone = [api.TopologyOptimizer.run(m, o, ctx=ctx) for m, o in jobs]
    with api.Server(slots=6, hbm_budget_bytes=8 * 10**9) as srv:
        ids = [srv.submit(m, o, keep_u=True) for m, o in jobs]
        srv.wait()
        for jid, ref in zip(ids, alone):
            r = srv.result(jid, u=True)
            assert r["info"]["state"] == "done", r["info"]["message"]
            assert [a.compliance for a in r["history"]] == [b.compliance for b in ref.snapshots]
            assert np.array_equal(r["physical"], ref.final_physical_density)
            assert np.array_equal(r["u"], ref.final_displacements)
