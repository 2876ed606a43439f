"""Seeded synthetic problems for the FEM + SIMP path.

No public dataset is involved: every grid, mask, load and density field is generated here from a recorded
seed (numpy PCG64). The shapes follow the reference's own test models (the cantilever of
tests/Mycel.Core.Tests/Optimization/OptimizationTests.cs:354-387) and the benchmark configurations:

* ``cantilever``       clamped at x=0, load on the tip bottom edge x=nx, z=0 (equal node areas)
* ``simp_cantilever_40x20x10``  8,000 Hex8 elements, E0=1, nu=0.3, Emin/E0=1e-9, total load -1 in z
* ``sphere_carved_box``  96x48x24 box with seeded spheres carved out to ~98,400 active elements, random
                        densities in [0.1, 1], face x=0 clamped, uniform -z traction of total 1 on face x=nx
* ``bridge``           four bottom-corner 8x8 node supports, total load 1 over a central 16x16 top patch
* ``batched_instances`` many uneven cantilever/bridge problems with several load cases each
* ``job_stream``       Poisson arrivals of optimisation jobs with log-uniform sizes
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from .model import FeMaterial, FeModel, GridSpec, LoadCase, OptimizerOptions, SurfacePatch


def cantilever(nx=30, ny=10, nz=4, h=1.0, e0=3000.0, nu=0.3, emin_ratio=1e-6, force=-1000.0,
               element_density=None) -> FeModel:
    """Cantilever of OptimizationTests.CreateCantileverModel: clamp x=0, load on nodes (nx, j, 0)."""
    g = GridSpec(nx, ny, nz, h)
    dom = np.ones(g.total_elements, dtype=np.uint8)
    fixed_nodes = [g.node_index(0, j, k) for k in range(nz + 1) for j in range(ny + 1)]
    fixed = FeModel.fix_dofs(fixed_nodes)
    tip = [g.node_index(nx, j, 0) for j in range(ny + 1)]
    patch = SurfacePatch(tip, [h * h] * len(tip))
    return FeModel(g, dom, FeMaterial(e0, nu, emin_ratio), fixed, [LoadCase(patch, (0.0, 0.0, force))],
                   element_density=element_density)


def v10_cantilever(target_elements: int, element_density: Optional[float] = None) -> FeModel:
    """The reference's V10 scaling benchmark model (FemValidationTests.cs:633-676): a solid 5d x d x d cantilever,
    nz = round(cbrt(target / 5)), h = 1, E0 = 3000, nu = 0.3 (Emin/E0 1e-6), every DOF of the x=0 nodes fixed,
    (0, 0, -1000) over all nodes of the x=nx face with area h^2 each; element_density: uniform density
    (the benchmark's 2 % perturbation uses 0.98), else 1."""
    nz = int(round(float(np.cbrt(target_elements / 5.0))))
    ny, nx = nz, 5 * nz
    g = GridSpec(nx, ny, nz, 1.0)
    dom = np.ones(g.total_elements, dtype=np.uint8)
    fixed = FeModel.fix_dofs([g.node_index(0, j, k) for k in range(nz + 1) for j in range(ny + 1)])
    tip = [g.node_index(nx, j, k) for k in range(nz + 1) for j in range(ny + 1)]
    patch = SurfacePatch(tip, [1.0] * len(tip))
    dens = None if element_density is None else np.full(g.total_elements, float(element_density))
    return FeModel(g, dom, FeMaterial(3000.0, 0.3), fixed, [LoadCase(patch, (0.0, 0.0, -1000.0))],
                   element_density=dens)


def simp_cantilever_40x20x10():
    """Plain FP64 SIMP cantilever: 40x20x10 unit voxels (8,000 elements), E0=1, nu=0.3, Emin=1e-9, p=3,
    volfrac=0.3, cone filter rmin=1.5, all DOFs fixed on x=0, total load -1 in z spread uniformly over the
    nodes of the edge x=40, z=0; PCG tolerance 1e-8, max 2,000 iterations; move 0.2; 30 iterations."""
    m = cantilever(40, 20, 10, 1.0, e0=1.0, nu=0.3, emin_ratio=1e-9, force=-1.0)
    opts = OptimizerOptions(volume_fraction=0.3, filter_radius_mm=1.5, penal=3.0, move_limit=0.2, max_iterations=30,
                            solver_tolerance_initial=1e-8, solver_tolerance_final=1e-8, solver_max_iterations=2000)
    return m, opts


def _face_connected_from_x0(active: np.ndarray) -> np.ndarray:
    """Keep the elements face-connected (6-neighbour) to the x=0 layer; active is (nz, ny, nx) bool."""
    try:
        from scipy import ndimage
    except ImportError:  # pragma: no cover - scipy is part of the environment; the loop below is the same rule
        ndimage = None
    if ndimage is not None:
        lab, _n = ndimage.label(active)  # default structure: 6-connectivity in 3-D
        roots = np.unique(lab[:, :, 0])
        roots = roots[roots > 0]
        return np.isin(lab, roots) & active
    keep = np.zeros_like(active)
    keep[:, :, 0] = active[:, :, 0]
    frontier = keep.copy()
    while frontier.any():
        grow = np.zeros_like(active)
        grow[1:, :, :] |= frontier[:-1, :, :]
        grow[:-1, :, :] |= frontier[1:, :, :]
        grow[:, 1:, :] |= frontier[:, :-1, :]
        grow[:, :-1, :] |= frontier[:, 1:, :]
        grow[:, :, 1:] |= frontier[:, :, :-1]
        grow[:, :, :-1] |= frontier[:, :, 1:]
        frontier = grow & active & ~keep
        keep |= frontier
    return keep


def exposed_face_patch(grid: GridSpec, domain: np.ndarray, face: str = "+x") -> SurfacePatch:
    """Tributary areas on an exposed box face: each exposed element face gives h^2/4 to its 4 corner nodes
    (the rule of src/Mycel.Core/Voxelization/SurfacePatchBuilder.cs:56-99)."""
    g = grid
    d = domain.reshape(g.nz, g.ny, g.nx) != 0
    area = {}
    q = 0.25 * float(np.float32(g.h)) ** 2
    if face == "+x":
        for iz in range(g.nz):
            for iy in range(g.ny):
                if d[iz, iy, g.nx - 1]:
                    for dj in (0, 1):
                        for dk in (0, 1):
                            n = g.node_index(g.nx, iy + dj, iz + dk)
                            area[n] = area.get(n, 0.0) + q
    else:
        raise ValueError(face)
    nodes = np.array(sorted(area), dtype=np.int32)
    return SurfacePatch(nodes, np.array([area[n] for n in nodes]))


def sphere_carved_box(nx=96, ny=48, nz=24, target_active=98_400, seed=2024, e0=1.0, nu=0.3, emin_ratio=1e-9,
                      rmin_sphere=2.0, rmax_sphere=5.0):
    """Box with seeded spheres carved out until about ``target_active`` elements stay active; densities uniform
    in [0.1, 1]; x=0 face clamped; uniform -z traction of total 1 on face x=nx."""
    rng = np.random.default_rng(seed)
    g = GridSpec(nx, ny, nz, 1.0)
    zz, yy, xx = np.meshgrid(np.arange(nz) + 0.5, np.arange(ny) + 0.5, np.arange(nx) + 0.5, indexing="ij")
    act = np.ones((nz, ny, nx), dtype=bool)
    while act.sum() > target_active:
        c = rng.uniform([0, 0, 0], [nx, ny, nz])
        r = rng.uniform(rmin_sphere, rmax_sphere)
        inside = (xx - c[0]) ** 2 + (yy - c[1]) ** 2 + (zz - c[2]) ** 2 <= r * r
        inside[:, :, 0] = False  # keep the clamped layer and the loaded layer solid
        inside[:, :, nx - 1] = False
        act &= ~inside
    act = _face_connected_from_x0(act)
    dom = act.reshape(-1).astype(np.uint8)
    dens = rng.uniform(0.1, 1.0, size=g.total_elements)
    fixed_nodes = [g.node_index(0, j, k) for k in range(nz + 1) for j in range(ny + 1)]
    fixed = FeModel.fix_dofs(fixed_nodes)
    patch = exposed_face_patch(g, dom, "+x")
    return FeModel(g, dom, FeMaterial(e0, nu, emin_ratio), fixed, [LoadCase(patch, (0.0, 0.0, -1.0))],
                   element_density=dens)


def bridge(nx=192, ny=96, nz=96, support=8, load_patch=16, e0=1.0, nu=0.3, emin_ratio=1e-9, force=-1.0,
           domain=None) -> FeModel:
    """Bridge: four bottom-corner support x support node patches fully fixed; total load ``force`` in z spread
    over a central load_patch x load_patch node patch on the top face (equal node areas)."""
    g = GridSpec(nx, ny, nz, 1.0)
    dom = np.ones(g.total_elements, dtype=np.uint8) if domain is None else np.asarray(domain, dtype=np.uint8)
    fixed_nodes = []
    for i0 in (0, nx + 1 - support):
        for j0 in (0, ny + 1 - support):
            for j in range(j0, j0 + support):
                for i in range(i0, i0 + support):
                    fixed_nodes.append(g.node_index(i, j, 0))
    fixed = FeModel.fix_dofs(sorted(fixed_nodes))
    ci, cj = nx // 2, ny // 2
    i0, j0 = ci - load_patch // 2, cj - load_patch // 2
    nodes = [g.node_index(i, j, nz) for j in range(j0, j0 + load_patch) for i in range(i0, i0 + load_patch)]
    patch = SurfacePatch(nodes, np.ones(len(nodes)))
    return FeModel(g, dom, FeMaterial(e0, nu, emin_ratio), fixed, [LoadCase(patch, (0.0, 0.0, force))])


def bridge_192x96x96():
    """Mixed-precision SIMP bridge: 192x96x96 (1,769,472 elements), volfrac=0.15, rmin=2.5, p=3, 50 iterations,
    warm-started PCG. Emin/E0 = 1e-9 (the harder case for FP32)."""
    m = bridge(192, 96, 96)
    opts = OptimizerOptions(volume_fraction=0.15, filter_radius_mm=2.5, penal=3.0, move_limit=0.2, max_iterations=50,
                            solver_tolerance_initial=1e-6, solver_tolerance_final=1e-6, solver_max_iterations=20000)
    return m, opts


@dataclass
class BatchedProblem:
    model: FeModel
    options: OptimizerOptions
    load_cases: List[LoadCase]


def batched_instances(count=48, seed=7, nx_range=(24, 128), nz_range=(8, 64), scale: float = 1.0):
    """Independent cantilever/bridge problems: nx in [24,128], ny = nx/2, nz in [8,64], 1-6 load cases of random
    unit direction on seeded 4x4 node patches of the free end, volfrac in [0.1,0.4], rmin in [1.2,3.0].
    ``scale`` shrinks the grids (for tests)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nx = max(4, int(round(rng.integers(nx_range[0], nx_range[1] + 1) * scale)))
        ny = max(2, nx // 2)
        nz = max(2, int(round(rng.integers(nz_range[0], nz_range[1] + 1) * scale)))
        kind = "bridge" if rng.random() < 0.5 else "cantilever"
        g = GridSpec(nx, ny, nz, 1.0)
        dom = np.ones(g.total_elements, dtype=np.uint8)
        ncase = int(rng.integers(1, 7))
        cases = []
        for _c in range(ncase):
            v = rng.normal(size=3)
            v /= np.linalg.norm(v)
            j0 = int(rng.integers(0, ny + 1 - 4 + 1)) if ny >= 3 else 0
            k0 = int(rng.integers(0, nz + 1 - 4 + 1)) if nz >= 3 else 0
            nodes = [g.node_index(nx, j, k) for k in range(k0, min(k0 + 4, nz + 1)) for j in range(j0, min(j0 + 4, ny + 1))]
            cases.append(LoadCase(SurfacePatch(nodes, np.ones(len(nodes))), tuple(v)))
        if kind == "cantilever":
            fixed_nodes = [g.node_index(0, j, k) for k in range(nz + 1) for j in range(ny + 1)]
        else:
            fixed_nodes = [g.node_index(i, j, 0) for i in (0, nx) for j in range(ny + 1)]
            fixed_nodes += [g.node_index(0, j, k) for k in range(nz + 1) for j in range(ny + 1)]
            fixed_nodes = sorted(set(fixed_nodes))
        fixed = FeModel.fix_dofs(fixed_nodes)
        model = FeModel(g, dom, FeMaterial(1.0, 0.3, 1e-9), fixed, cases)
        opts = OptimizerOptions(volume_fraction=float(rng.uniform(0.1, 0.4)), filter_radius_mm=float(rng.uniform(1.2, 3.0)),
                                penal=3.0, move_limit=0.2, max_iterations=1, solver_tolerance_initial=1e-6,
                                solver_tolerance_final=1e-6, solver_max_iterations=20000)
        out.append(BatchedProblem(model, opts, cases))
    return out


def job_stream(n_jobs=500, rate=20.0, seed=11, min_elems=8_000, max_elems=1_000_000, iters=(20, 60)):
    """Poisson arrivals (``rate`` jobs/s) of SIMP jobs with log-uniform element counts in [min, max] and
    20-60 iterations each. Returns a list of (arrival_s, nx, ny, nz, n_iters, seed)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for j in range(n_jobs):
        t += rng.exponential(1.0 / rate)
        ne = float(np.exp(rng.uniform(np.log(min_elems), np.log(max_elems))))
        nz = max(4, int(round((ne / 8.0) ** (1.0 / 3.0))))
        ny = 2 * nz
        nx = max(8, int(round(ne / (ny * nz))))
        jobs.append((t, nx, ny, nz, int(rng.integers(iters[0], iters[1] + 1)), int(rng.integers(0, 2**31 - 1))))
    return jobs


def served_job(nx: int, ny: int, nz: int, n_iters: int, seed: int, precision: str = "mixed", tol: float = 1e-6):
    """One job of the served stream: a box with seeded spheres (radius 2-5 voxels, about 15 % of the volume)
    carved out and the part face-connected to x=0 kept; all DOFs of the active x=0 nodes fixed; 1-3 load cases
    of random unit direction on seeded 4x4 node patches of the x=nx face (active nodes, equal areas);
    volfrac in [0.1, 0.4], rmin in [1.2, 3.0], n_iters SIMP iterations, warm-started PCG to relative residual
    ``tol`` in every iteration (as the 192x96x96 bridge). Returns (model, options)."""
    rng = np.random.default_rng(seed)
    g = GridSpec(nx, ny, nz, 1.0)
    act = np.ones((nz, ny, nx), dtype=bool)
    target = 0.85 * act.size
    n_act = act.size
    for _ in range(100_000):
        if n_act <= target:
            break
        c = rng.uniform([0, 0, 0], [nx, ny, nz])
        r = rng.uniform(2.0, 5.0)
        lo = [max(0, int(np.floor(c[a] - r))) for a in range(3)]
        hi = [min(n, int(np.ceil(c[a] + r)) + 1) for a, n in enumerate((nx, ny, nz))]
        zz, yy, xx = np.meshgrid(np.arange(lo[2], hi[2]) + 0.5, np.arange(lo[1], hi[1]) + 0.5,
                                 np.arange(lo[0], hi[0]) + 0.5, indexing="ij")
        inside = (xx - c[0]) ** 2 + (yy - c[1]) ** 2 + (zz - c[2]) ** 2 <= r * r
        inside &= (xx > 1.0) & (xx < nx - 1.0)  # keep the clamped layer x=0 and the loaded layer x=nx-1
        box = act[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
        n_act -= int((box & inside).sum())
        box &= ~inside
    act = _face_connected_from_x0(act)
    dom = act.reshape(-1).astype(np.uint8)
    node_act = np.zeros((nz + 1, ny + 1, nx + 1), dtype=bool)
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                node_act[dz:dz + nz, dy:dy + ny, dx:dx + nx] |= act
    fixed_nodes = [g.node_index(0, j, k) for k in range(nz + 1) for j in range(ny + 1) if node_act[k, j, 0]]
    cases = []
    for _c in range(int(rng.integers(1, 4))):
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        j0 = int(rng.integers(0, max(1, ny - 2)))
        k0 = int(rng.integers(0, max(1, nz - 2)))
        nodes = [g.node_index(nx, j, k) for k in range(k0, min(k0 + 4, nz + 1)) for j in range(j0, min(j0 + 4, ny + 1))
                 if node_act[k, j, nx]]
        if not nodes:
            nodes = [g.node_index(nx, j, k) for k in range(nz + 1) for j in range(ny + 1) if node_act[k, j, nx]]
        cases.append(LoadCase(SurfacePatch(nodes, np.ones(len(nodes))), tuple(float(x) for x in v)))
    model = FeModel(g, dom, FeMaterial(1.0, 0.3, 1e-9), FeModel.fix_dofs(fixed_nodes), cases)
    opts = OptimizerOptions(volume_fraction=float(rng.uniform(0.1, 0.4)), filter_radius_mm=float(rng.uniform(1.2, 3.0)),
                            penal=3.0, move_limit=0.2, max_iterations=int(n_iters), solver_tolerance_initial=tol,
                            solver_tolerance_final=tol, solver_max_iterations=20000, precision=precision)
    return model, opts


def saddle_density(nx, ny, nz, seed=0, p=0.45):
    """Seeded float32 density whose 0.5-level set is full of face saddles and corner kisses (the hard case of
    the iso-surface's well-composedness passes): uniform values, a fraction p of them above 0.5."""
    rng = np.random.default_rng(seed)
    v = rng.random(nx * ny * nz).astype(np.float32)
    return np.where(rng.random(nx * ny * nz) < p, 0.5 + 0.5 * v, 0.5 * v).astype(np.float32)
