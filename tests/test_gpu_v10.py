"""The plain FP64 path on the reference's V10 scaling benchmark (FemValidationTests.cs:633-726): the
reference's published PCG iteration counts (docs/STEP3_BENCH.md:25-26) and the oracle's u, bit for bit."""
import numpy as np
import pytest

from mycel_b200 import api, workloads as W
from mycel_b200.model import StaticAnalysisOptions

from test_oracle_pins import V10_PUBLISHED, v10_counts

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("target,elements", [(50_000, 53_240), (100_000, 98_415)])
def test_v10_counts_and_bits(oracle, ctx, target, elements):
    oracle.set_modes(0, threads=8)
    m0, ref = v10_counts(oracle, target)
    assert m0.total_elements == elements
    mp = W.v10_cantilever(target, 0.98)
    c4 = api.StaticAnalysis.run(m0, StaticAnalysisOptions(tolerance=1e-4), ctx)
    w4 = api.StaticAnalysis.run(mp, StaticAnalysisOptions(tolerance=1e-4, warm_start_displacements=c4.u), ctx)
    cp = api.StaticAnalysis.run(mp, StaticAnalysisOptions(tolerance=1e-4), ctx)
    c6 = api.StaticAnalysis.run(m0, StaticAnalysisOptions(tolerance=1e-6), ctx)
    got = (c4, w4, cp, c6)
    assert tuple(r.solver_info.iterations for r in got) == V10_PUBLISHED[elements]
    for g, r in zip(got, ref):
        assert np.array_equal(g.u, r.u)
        assert g.compliance == r.compliance


def test_sphere_carved_static_solve_bit_exact(oracle, ctx):
    # the single FP64 FEA solve at the README's V10 scale: 96x48x24 box carved by seeded spheres to about
    # 98,400 active elements, densities in [0.1, 1], x=0 clamped, -z traction of total 1 on x=96, rel tol 1e-8
    oracle.set_modes(0, threads=8)
    m = W.sphere_carved_box()
    ref = oracle.static_run(m, 1e-8, 20_000)
    got = api.StaticAnalysis.run(m, StaticAnalysisOptions(tolerance=1e-8, max_iterations=20_000), ctx)
    assert got.solver_info.iterations == ref.solver_info.iterations
    assert got.solver_info.final_residual == ref.solver_info.final_residual
    assert np.array_equal(got.u, ref.u)
    assert np.array_equal(got.reactions, ref.reactions)
    assert got.compliance == ref.compliance and got.max_displacement == ref.max_displacement
