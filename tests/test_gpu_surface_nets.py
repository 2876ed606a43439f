"""Surface Nets on the device (mycel_surface_nets) against the oracle's sequential restatement of
SurfaceNetsExtractor.Extract: identical vertex positions (bit for bit), identical triangle indices and order,
and the same well-composedness passes and resolutions, on the reference tests' fields, border and degenerate
cases, and saddle-rich fields that drive several passes of the wavefront-scheduled well-composedness kernel."""
import numpy as np
import pytest

from mycel_b200 import api
from mycel_b200.model import ArgumentError, GridSpec
from meshtools import saddle_field, sphere_field, topology

pytestmark = pytest.mark.gpu


def _same(oracle, ctx, nx, ny, nz, dens, h=1.0, origin=(0.0, 0.0, 0.0), thr=0.5):
    ref_pos, ref_idx, info = oracle.surface_nets(nx, ny, nz, dens, h=h, origin=origin, threshold=thr)
    m = api.SurfaceNetsExtractor.extract(GridSpec(nx, ny, nz, h, origin), dens, thr, ctx=ctx)
    assert m.positions.shape == ref_pos.shape and m.indices.shape == ref_idx.shape
    assert np.array_equal(m.positions.view(np.uint32), ref_pos.view(np.uint32))
    assert np.array_equal(m.indices, ref_idx)
    assert (m.passes, m.changes) == (info["passes"], info["changes"])
    return m


def test_sphere_matches_oracle(oracle, ctx):
    m = _same(oracle, ctx, 32, 32, 32, sphere_field(32, 32, 32, [(16, 16, 16)], 12.0))
    op, nm, ne, comps = topology(m.indices)
    assert (op, nm, comps) == (0, 0, 1) and m.vertex_count - ne + m.triangle_count == 2


def test_two_spheres_and_border_cube_match_oracle(oracle, ctx):
    _same(oracle, ctx, 40, 20, 20, sphere_field(40, 20, 20, [(10, 10, 10), (30, 10, 10)], 6.0))
    _same(oracle, ctx, 10, 10, 10, np.ones(1000, dtype=np.float32), h=2.0, origin=(10.0, 20.0, 30.0))


@pytest.mark.parametrize("shape,seed", [((14, 11, 9), 3), ((33, 17, 9), 5), ((1, 7, 5), 1), ((20, 1, 6), 2),
                                        ((9, 8, 1), 4), ((64, 40, 24), 7)])
def test_saddle_fields_match_oracle(oracle, ctx, shape, seed):
    nx, ny, nz = shape
    m = _same(oracle, ctx, nx, ny, nz, saddle_field(nx, ny, nz, seed=seed), thr=0.5)
    if min(shape) > 1:
        assert m.changes > 0


def test_threshold_and_empty_fields(oracle, ctx):
    d = sphere_field(24, 20, 16, [(12, 10, 8)], 6.5)
    _same(oracle, ctx, 24, 20, 16, d, thr=0.3)
    _same(oracle, ctx, 24, 20, 16, d, thr=0.8)
    m = _same(oracle, ctx, 6, 5, 4, np.zeros(120, dtype=np.float32))
    assert m.vertex_count == 0 and m.triangle_count == 0


def test_short_density_is_an_argument_error(ctx):
    with pytest.raises(ArgumentError, match="smaller than grid element count"):
        api.SurfaceNetsExtractor.extract(GridSpec(4, 4, 4), np.zeros(63, dtype=np.float32), ctx=ctx)


@pytest.mark.parametrize("iters", [1, 3, 7])
def test_taubin_matches_oracle(oracle, ctx, iters):
    d = sphere_field(40, 20, 20, [(10, 10, 10), (30, 10, 10)], 6.0)
    m = api.SurfaceNetsExtractor.extract(GridSpec(40, 20, 20), d, 0.5, ctx=ctx)
    sm = api.TaubinSmoother.smooth(m, iters, ctx=ctx)
    ref = oracle.taubin_smooth(m.positions, m.indices, iters)
    assert np.array_equal(sm.positions.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(sm.indices, m.indices)


def test_taubin_on_saddle_mesh_and_bad_index(oracle, ctx):
    d = saddle_field(20, 14, 10, seed=9)
    m = api.SurfaceNetsExtractor.extract(GridSpec(20, 14, 10), d, 0.5, ctx=ctx)
    sm = api.TaubinSmoother.smooth(m, 3, ctx=ctx)
    assert np.array_equal(sm.positions.view(np.uint32), oracle.taubin_smooth(m.positions, m.indices, 3).view(np.uint32))
    bad = api.IndexedMesh(m.positions, np.concatenate([m.indices[:-3], [0, 1, m.vertex_count]]).astype(np.int32))
    with pytest.raises(ArgumentError, match="out of range"):
        api.TaubinSmoother.smooth(bad, 3, ctx=ctx)


def test_session_mesh_equals_host_extraction(oracle, ctx):
    """The preview path: a SIMP session's iso-surface from its device-resident density equals the extraction
    of the density it reads back (and the oracle's)."""
    from mycel_b200 import workloads as W
    m, o = W.simp_cantilever_40x20x10()
    pr = api.Problem(m, ctx)
    s = api.SimpSession(pr, o.replace(max_iterations=6))
    for _ in range(6):
        s.step()
    mesh = s.surface_mesh(0.5)
    rho = s.read(u=False, densities=True)["physical"]
    g = m.grid
    ref = _same(oracle, ctx, g.nx, g.ny, g.nz, rho, h=float(g.h))
    assert np.array_equal(mesh.positions.view(np.uint32), ref.positions.view(np.uint32))
    assert np.array_equal(mesh.indices, ref.indices) and mesh.triangle_count > 0
    s.close()
    pr.close()
