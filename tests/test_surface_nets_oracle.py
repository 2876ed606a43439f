"""Surface Nets oracle (CPU restatement of SurfaceNetsExtractor.Extract) pinned by the reference's own
iso-surface tests (Step6Tests.cs T1 and T2): a closed 2-manifold sphere with Euler characteristic 2 and volume
within 3 %, two disjoint spheres (2 components, Euler 4), and a border-touching cube closed by the padding with
its box in world coordinates; plus the well-composedness passes on a saddle-rich field."""
import math

import numpy as np

from meshtools import saddle_field, signed_volume, sphere_field, topology


def test_sphere_closed_manifold_euler2_volume(oracle):
    n = 32
    pos, idx, info = oracle.surface_nets(n, n, n, sphere_field(n, n, n, [(16, 16, 16)], 12.0))
    assert len(pos) > 0 and len(idx) > 0
    op, nm, ne, comps = topology(idx)
    assert (op, nm, comps) == (0, 0, 1)
    assert len(pos) - ne + len(idx) // 3 == 2
    exact = 4.0 / 3.0 * math.pi * 12.0 ** 3
    assert abs(abs(signed_volume(pos, idx)) - exact) / exact < 0.03


def test_two_spheres_and_border_cube(oracle):
    pos, idx, _ = oracle.surface_nets(40, 20, 20, sphere_field(40, 20, 20, [(10, 10, 10), (30, 10, 10)], 6.0))
    op, nm, ne, comps = topology(idx)
    assert (op, nm, comps) == (0, 0, 2)
    assert len(pos) - ne + len(idx) // 3 == 4
    cube = np.ones(1000, dtype=np.float32)
    pos, idx, _ = oracle.surface_nets(10, 10, 10, cube, h=2.0, origin=(10.0, 20.0, 30.0))
    op, nm, ne, comps = topology(idx)
    assert (op, nm, comps) == (0, 0, 1)
    assert len(pos) - ne + len(idx) // 3 == 2
    lo, hi = pos.min(axis=0), pos.max(axis=0)
    assert np.all(np.abs(lo - [10, 20, 30]) < 1.5) and np.all(np.abs(hi - [30, 40, 50]) < 1.5)


def test_empty_and_full_fields(oracle):
    pos, idx, info = oracle.surface_nets(5, 4, 3, np.zeros(60, dtype=np.float32))
    assert len(pos) == 0 and len(idx) == 0 and info["passes"] == 1


def test_saddle_field_is_made_well_composed(oracle):
    """Saddles and corner kisses are resolved (changes > 0) and the surface is then free of open and
    non-manifold edges."""
    pos, idx, info = oracle.surface_nets(14, 11, 9, saddle_field(14, 11, 9, seed=3))
    assert info["changes"] > 0 and info["passes"] >= 2
    op, nm, _, _ = topology(idx)
    assert op == 0


def test_taubin_keeps_topology_and_volume(oracle):
    """The reference's export test (Step6Tests T3) smooths the extracted sphere with 3 Taubin iterations and
    requires a watertight result whose volume is kept: topology unchanged, volume within 1 %, and the
    staircase reduced (radial spread of the vertices shrinks)."""
    n = 24
    pos, idx, _ = oracle.surface_nets(n, n, n, sphere_field(n, n, n, [(12, 12, 12)], 8.0))
    sm = oracle.taubin_smooth(pos, idx, 3)
    assert sm.shape == pos.shape and not np.array_equal(sm, pos)
    v0, v1 = signed_volume(pos, idx), signed_volume(sm, idx)
    assert abs(v1 - v0) / abs(v0) < 0.01
    r0 = np.linalg.norm(pos - 12.0, axis=1)
    r1 = np.linalg.norm(sm - 12.0, axis=1)
    assert r1.std() < r0.std()
    assert np.array_equal(oracle.taubin_smooth(pos, idx, 0), pos)
