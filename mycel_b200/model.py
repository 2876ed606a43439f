"""Host-side mirror of Mycel.Core's call-surface types for the FEM + SIMP path.

These are plain data holders with the same names, fields and defaults as the C# records and classes they
mirror, so that code written against Mycel.Core reads the same here:

* ``GridSpec``            src/Mycel.Core/Voxelization/GridSpec.cs:11-204 (node/element/DOF indexing)
* ``FeMaterial``          src/Mycel.Core/Fem/FeMaterial.cs:11-16
* ``SurfacePatch``        src/Mycel.Core/Voxelization/SurfacePatch.cs:25-49 (nodes + tributary areas)
* ``LoadCase``            src/Mycel.Core/Fem/LoadCase.cs:10-19 (``TotalForce`` is a float Vector3)
* ``FeModel``             src/Mycel.Core/Fem/FeModel.cs:11-256 (constructor validation, ``FixDofs`` helpers)
* ``StaticAnalysisOptions`` src/Mycel.Core/Fem/StaticAnalysis.cs:8-17
* ``OptimizerOptions``    src/Mycel.Core/Optimization/OptimizerOptions.cs:5-26
* ``IterationSnapshot``   src/Mycel.Core/Optimization/IterationSnapshot.cs:5-31
* ``PcgResult``           src/Mycel.Core/Fem/PcgResult.cs:5-14

Errors are raised with the same exception classes the reference throws (``ArgumentError`` for
ArgumentException/ArgumentOutOfRangeException, ``InvalidOperationError`` for InvalidOperationException).
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np


class MycelError(RuntimeError):
    """Base class of errors raised through the C ABI."""

    status = 0


class ArgumentError(MycelError, ValueError):
    """ArgumentException / ArgumentOutOfRangeException in the reference."""

    status = 1


class InvalidOperationError(MycelError):
    """InvalidOperationException in the reference (under-constrained model, non-convergence)."""

    status = 9


class CancelledError(MycelError):
    status = 5


class DeviceError(MycelError):
    status = 7


class TimeoutError_(MycelError):
    status = 6


class OutOfMemoryError(MycelError):
    status = 8


@dataclass(frozen=True)
class GridSpec:
    """Regular grid of cubic Hex8 voxels: e = ix + Nx(iy + Ny iz), n = i + (Nx+1)(j + (Ny+1)k), dof = 3n + c."""

    nx: int
    ny: int
    nz: int
    h: float = 1.0
    origin: tuple = (0.0, 0.0, 0.0)

    def __post_init__(self):
        if not (np.float32(self.h) > 0):
            raise ArgumentError("Voxel pitch must be positive.")
        if self.nx <= 0 or self.ny <= 0 or self.nz <= 0:
            raise ArgumentError("Grid dimensions must be strictly positive.")

    @property
    def total_elements(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def total_nodes(self) -> int:
        return (self.nx + 1) * (self.ny + 1) * (self.nz + 1)

    @property
    def total_dofs(self) -> int:
        return 3 * self.total_nodes

    def element_index(self, ix: int, iy: int, iz: int) -> int:
        if not (0 <= ix < self.nx and 0 <= iy < self.ny and 0 <= iz < self.nz):
            raise ArgumentError(f"Element coordinates ({ix}, {iy}, {iz}) out of bounds.")
        return ix + self.nx * (iy + self.ny * iz)

    def node_index(self, i: int, j: int, k: int) -> int:
        if not (0 <= i <= self.nx and 0 <= j <= self.ny and 0 <= k <= self.nz):
            raise ArgumentError(f"Node coordinates ({i}, {j}, {k}) out of bounds.")
        return i + (self.nx + 1) * (j + (self.ny + 1) * k)

    def inverse_element_index(self, e: int):
        nxny = self.nx * self.ny
        iz, rem = divmod(e, nxny)
        iy, ix = divmod(rem, self.nx)
        return ix, iy, iz

    def inverse_node_index(self, n: int):
        nx1 = self.nx + 1
        k, rem = divmod(n, nx1 * (self.ny + 1))
        j, i = divmod(rem, nx1)
        return i, j, k


@dataclass(frozen=True)
class FeMaterial:
    e0: float
    nu: float
    emin_ratio: float = 1e-6

    @property
    def emin(self) -> float:
        return self.e0 * self.emin_ratio


@dataclass
class SurfacePatch:
    nodes: np.ndarray
    node_area: np.ndarray

    def __post_init__(self):
        self.nodes = np.ascontiguousarray(np.asarray(self.nodes, dtype=np.int32).reshape(-1))
        self.node_area = np.ascontiguousarray(np.asarray(self.node_area, dtype=np.float64).reshape(-1))
        if self.nodes.shape != self.node_area.shape:
            raise ArgumentError("SurfacePatch nodes and node areas must have the same length.")

    @property
    def node_count(self) -> int:
        return int(self.nodes.size)


@dataclass
class LoadCase:
    patch: SurfacePatch
    total_force: tuple  # (fx, fy, fz), stored as float32 like System.Numerics.Vector3

    def __post_init__(self):
        self.total_force = tuple(float(np.float32(v)) for v in self.total_force)


class FeModel:
    """Grid + domain mask + material + fixed DOFs + loads + densities (FeModel.cs:43-184)."""

    def __init__(self, grid: GridSpec, domain, material: FeMaterial, fixed_dofs, loads: Optional[Sequence[LoadCase]] = None,
                 element_density=None, penal: float = 3.0):
        self.grid = grid
        self.domain = np.ascontiguousarray(np.asarray(domain, dtype=np.uint8).reshape(-1))
        self.material = material
        self.fixed_dofs = np.ascontiguousarray(np.asarray(fixed_dofs if fixed_dofs is not None else [], dtype=np.int64).reshape(-1))
        self.penal = float(penal)
        if self.domain.size != grid.total_elements:
            raise ArgumentError(
                f"Domain array length ({self.domain.size}) does not match Grid TotalElements ({grid.total_elements}).")
        self.loads: List[LoadCase] = list(loads) if loads is not None else []
        if element_density is not None:
            d = np.asarray(element_density, dtype=np.float64).reshape(-1)
            if d.size != grid.total_elements:
                raise ArgumentError(
                    f"ElementDensity length ({d.size}) must match TotalElements ({grid.total_elements}).")
            self.element_density = d.copy()
        else:
            self.element_density = np.ones(grid.total_elements, dtype=np.float64)
        bad = (self.fixed_dofs < 0) | (self.fixed_dofs >= grid.total_dofs)
        if bad.any():
            dof = int(self.fixed_dofs[bad][0])
            raise ArgumentError(f"Fixed DOF {dof} is out of bounds [0, {grid.total_dofs - 1}].")
        self.fixed_dofs = self.fixed_dofs.astype(np.int32)
        e = np.nonzero(self.domain)[0]
        self.active_elements = e.astype(np.int32)

    @property
    def total_elements(self) -> int:
        return self.grid.total_elements

    @property
    def total_nodes(self) -> int:
        return self.grid.total_nodes

    @property
    def total_dofs(self) -> int:
        return self.grid.total_dofs

    @property
    def active_element_count(self) -> int:
        return int(self.active_elements.size)

    def active_nodes_mask(self) -> np.ndarray:
        g = self.grid
        d = self.domain.reshape(g.nz, g.ny, g.nx) != 0
        a = np.zeros((g.nz + 1, g.ny + 1, g.nx + 1), dtype=bool)
        for dz in (0, 1):
            for dy in (0, 1):
                for dx in (0, 1):
                    a[dz:dz + g.nz, dy:dy + g.ny, dx:dx + g.nx] |= d
        return a.reshape(-1)

    @staticmethod
    def fix_dofs(nodes, fix_x: bool = True, fix_y: bool = True, fix_z: bool = True) -> np.ndarray:
        """FeModel.FixDofs(nodes, fixX, fixY, fixZ) (FeModel.cs:189-200)."""
        comps = [c for c, f in enumerate((fix_x, fix_y, fix_z)) if f]
        nodes = np.asarray(list(nodes), dtype=np.int64).reshape(-1)
        out = (3 * nodes[:, None] + np.asarray(comps, dtype=np.int64)[None, :]).reshape(-1)
        return out.astype(np.int32)


@dataclass
class StaticAnalysisOptions:
    tolerance: float = 1e-6
    max_iterations: int = 5000
    warm_start_displacements: Optional[np.ndarray] = None
    throw_on_non_convergence: bool = True
    # "fp64" (the plain drop-in), "mixed" (FP32 inner Jacobi-PCG + FP64 refinement), "fp64f" (factorised FP64
    # operator), "mg" (FP64 flexible CG with an FP32 multigrid V-cycle), "mixed-mg" (that iteration in FP32 inside
    # FP64 refinement)
    precision: str = "fp64"


@dataclass
class PcgResult:
    iterations: int = 0
    final_residual: float = 0.0
    converged: bool = False
    elapsed_ms: float = 0.0
    message: Optional[str] = None
    refinement_steps: int = 0
    inner_iterations: int = 0     # mixed form: FP32 inner iterations
    fallback_iterations: int = 0  # mixed form: FP64 iterations that finished a stalled solve


@dataclass
class StaticAnalysisResult:
    u: np.ndarray
    compliance: float
    reactions: Optional[np.ndarray]
    max_displacement: float
    solver_info: PcgResult
    von_mises_per_element: Optional[np.ndarray] = None


@dataclass
class OptimizerOptions:
    volume_fraction: float = 0.4
    filter_radius_mm: float = 2.0
    penal: float = 3.0
    move_limit: float = 0.2
    max_iterations: int = 200
    solver_tolerance_initial: float = 1e-4
    solver_tolerance_final: float = 1e-6
    solver_max_iterations: int = 5000
    emin_ratio: float = 1e-6  # present in the reference's record but not read by the optimiser
    continuation: bool = False
    enable_heaviside: bool = False
    rng_seed: int = 42
    rho_min: float = 1e-3
    passive_mask: Optional[np.ndarray] = None
    protect_boundary_hinges: bool = True
    initial_density: Optional[np.ndarray] = None
    start_iteration: int = 1
    warm_start_displacements: Optional[np.ndarray] = None
    enforce_minimum_filter_radius: bool = True
    precision: str = "fp64"  # solver form, as for StaticAnalysisOptions.precision
    # Load cases: False sums them into one right-hand side (FeModel.AssembleForces, the reference's behaviour);
    # True solves each case on the shared stiffness (its own warm start), minimises the sum of the cases'
    # compliances, sums the sensitivities over the cases in case order and reports u as the sum of the cases'
    # displacements. An extension: the reference has no multi-load objective.
    separate_load_cases: bool = False

    def replace(self, **kw) -> "OptimizerOptions":
        return dataclasses.replace(self, **kw)


@dataclass
class IterationSnapshot:
    iteration: int
    compliance: float
    volume_fraction: float
    max_change: float
    grey_level: float
    solver_iterations: int
    solver_residual: float
    max_displacement: float
    solve_ms: float = 0.0
    sensitivity_ms: float = 0.0
    filter_ms: float = 0.0
    update_ms: float = 0.0
    total_ms: float = 0.0
    physical_density: Optional[np.ndarray] = None
    design_density: Optional[np.ndarray] = None


@dataclass
class TopologyOptimizationResult:
    converged: bool
    total_iterations: int
    snapshots: List[IterationSnapshot]
    final_compliance: float
    final_volume_fraction: float
    final_physical_density: np.ndarray
    final_design_density: np.ndarray
    final_displacements: np.ndarray
    warnings: List[str] = field(default_factory=list)

    @property
    def final_snapshot(self) -> IterationSnapshot:
        return self.snapshots[-1]
