"""Model builders that mirror the reference's test fixtures (tests/Mycel.Core.Tests/**)."""
import numpy as np

from mycel_b200.model import FeMaterial, FeModel, GridSpec, LoadCase, SurfacePatch


def bar_model(length, width, height, h, e0, nu):
    """FemValidationTests.CreateBarModel (FemValidationTests.cs:13-59): clamp x=0, tip patch on x=L."""
    nx, ny, nz = int(round(length / h)), int(round(width / h)), int(round(height / h))
    g = GridSpec(nx, ny, nz, h)
    fixed = FeModel.fix_dofs([g.node_index(0, j, k) for k in range(nz + 1) for j in range(ny + 1)])
    tn, ta = [], []
    for k in range(nz + 1):
        for j in range(ny + 1):
            tn.append(g.node_index(nx, j, k))
            dy = 0.5 * h if j in (0, ny) else h
            dz = 0.5 * h if k in (0, nz) else h
            ta.append(dy * dz)
    model = FeModel(g, np.ones(g.total_elements), FeMaterial(e0, nu), fixed)
    return model, SurfacePatch(tn, ta)


def tiny_test_model(nx=6, ny=4, nz=3, h=1.0, e0=3000.0, nu=0.3, emin_ratio=1e-6):
    """OptimizationTests.CreateTinyTestModel (OptimizationTests.cs:18-66): two point loads on x=nx."""
    g = GridSpec(nx, ny, nz, h)
    fixed = FeModel.fix_dofs([g.node_index(0, j, k) for k in range(nz + 1) for j in range(ny + 1)])
    p1 = SurfacePatch([g.node_index(nx, 0, 0)], [h * h])
    p2 = SurfacePatch([g.node_index(nx, ny, nz)], [h * h])
    return FeModel(g, np.ones(g.total_elements), FeMaterial(e0, nu, emin_ratio), fixed,
                   [LoadCase(p1, (0, 0, -100.0)), LoadCase(p2, (50.0, -30.0, 0))])


def l_shape_domain(nx=8, ny=6, nz=5):
    """T2 L-shaped domain (OptimizationTests.cs:216-233)."""
    g = GridSpec(nx, ny, nz, 1.0)
    d = np.zeros(g.total_elements, dtype=np.uint8)
    for iz in range(nz):
        for iy in range(ny):
            for ix in range(nx):
                if ix < nx // 2 or iy < ny // 2:
                    d[ix + nx * (iy + ny * iz)] = 1
    return g, d


def underconstrained_model():
    """V12 (FemValidationTests.cs:844-869): six fixed DOFs on one line, rotation about z free."""
    g = GridSpec(4, 4, 4, 1.0)
    fixed = FeModel.fix_dofs([g.node_index(0, 0, 0), g.node_index(0, 0, 4)])
    patch = SurfacePatch([g.node_index(4, 0, 2)], [1.0])
    return FeModel(g, np.ones(64), FeMaterial(1000.0, 0.3), fixed, [LoadCase(patch, (0, 100.0, 0))])


def carved_model(nx, ny, nz, seed=3, frac=0.2, emin_ratio=1e-9):
    """Cantilever with a seeded random void pattern (keeps x=0 and x=nx-1 layers solid)."""
    rng = np.random.default_rng(seed)
    g = GridSpec(nx, ny, nz, 1.0)
    dom = (rng.random((nz, ny, nx)) > frac)
    dom[:, :, 0] = True
    dom[:, :, -1] = True
    from mycel_b200.workloads import _face_connected_from_x0
    dom = _face_connected_from_x0(dom).reshape(-1).astype(np.uint8)
    fixed = FeModel.fix_dofs([g.node_index(0, j, k) for k in range(nz + 1) for j in range(ny + 1)])
    tip = [g.node_index(nx, j, 0) for j in range(ny + 1)]
    dens = rng.uniform(0.1, 1.0, g.total_elements)
    return FeModel(g, dom, FeMaterial(1.0, 0.3, emin_ratio), fixed,
                   [LoadCase(SurfacePatch(tip, np.ones(len(tip))), (0.3, -0.2, -1.0))], element_density=dens)
