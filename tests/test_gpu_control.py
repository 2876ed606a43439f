"""TopologyOptimizer.Run's control surface through mycel_simp_run: the progress callback
(IProgress<IterationSnapshot>, TopologyOptimizer.cs:341-347), cancellation (CancellationToken, :169-172) and
pause / resume / stop (IterationController.CheckAndBlock, IterationController.cs:9-65). Cancelling ends the loop
between iterations with the state of the last completed one, as the reference's `break` does."""
import threading
import time

import numpy as np
import pytest

from mycel_b200 import api, workloads as W
from mycel_b200.model import OptimizerOptions

pytestmark = pytest.mark.gpu


def _problem():
    m = W.cantilever(24, 8, 6)
    o = OptimizerOptions(volume_fraction=0.35, filter_radius_mm=1.5, max_iterations=8,
                         solver_tolerance_initial=1e-6, solver_tolerance_final=1e-8)
    return m, o


def test_progress_reports_every_iteration(ctx):
    m, o = _problem()
    seen = []
    res = api.TopologyOptimizer.run(m, o, progress=lambda s: seen.append(s), ctx=ctx)
    assert [s.iteration for s in seen] == list(range(1, res.total_iterations + 1))
    for a, b in zip(seen, res.snapshots):
        assert a.compliance == b.compliance and a.max_change == b.max_change
        assert a.physical_density.shape == (m.total_elements,) and a.design_density.dtype == np.float32
    # the last report carries the final densities
    assert np.array_equal(seen[-1].physical_density, res.final_physical_density)


def test_stop_from_the_callback_ends_after_that_iteration(ctx):
    m, o = _problem()
    full = api.TopologyOptimizer.run(m, o, ctx=ctx)
    ctl = api.IterationController()
    seen = []

    def cb(s):
        seen.append(s.iteration)
        if s.iteration == 3:
            ctl.stop()

    res = api.TopologyOptimizer.run(m, o, progress=cb, controller=ctl, ctx=ctx)
    assert res.total_iterations == 3 and seen == [1, 2, 3]
    # the first three iterations are the uncancelled run's
    for a, b in zip(res.snapshots, full.snapshots[:3]):
        assert a.compliance == b.compliance
    assert not res.converged


def test_pause_blocks_between_iterations_until_resumed(ctx):
    m, o = _problem()
    ctl = api.IterationController()
    ctl.pause()
    seen = []
    out = {}

    def run():
        out["res"] = api.TopologyOptimizer.run(m, o, progress=lambda s: seen.append(s.iteration), controller=ctl,
                                               ctx=api.Context(0))

    th = threading.Thread(target=run)
    th.start()
    time.sleep(1.0)
    assert seen == []  # paused before the first iteration
    ctl.resume()
    th.join(timeout=120)
    assert not th.is_alive()
    assert out["res"].total_iterations == o.max_iterations and seen == list(range(1, o.max_iterations + 1))


def test_stop_while_paused_ends_without_iterating(ctx):
    m, o = _problem()
    ctl = api.IterationController()
    ctl.pause()
    out = {}
    th = threading.Thread(target=lambda: out.setdefault(
        "res", api.TopologyOptimizer.run(m, o, controller=ctl, ctx=api.Context(0))))
    th.start()
    time.sleep(0.5)
    ctl.stop()
    th.join(timeout=60)
    assert not th.is_alive()
    assert out["res"].total_iterations == 0
