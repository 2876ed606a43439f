"""Mycel.Core-shaped host interface over the C ABI (the Python side of the drop-in boundary).

``StaticAnalysis.run`` and ``TopologyOptimizer.run`` take the same inputs and return the same results as the
reference's ``StaticAnalysis.Run`` (src/Mycel.Core/Fem/StaticAnalysis.cs:35) and ``TopologyOptimizer.Run``
(src/Mycel.Core/Optimization/TopologyOptimizer.cs:16), raising the same error classes. The kernel-level methods
of ``Problem`` mirror FemOperator / PcgSolver / DensityFilter / SensitivityAnalysis / OcOptimizer.
All arithmetic runs in libmycel_b200.so on the GPU.
"""
from __future__ import annotations

import ctypes as C
import threading
import weakref
from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import _lib as L
from .model import (ArgumentError, CancelledError, DeviceError, FeModel, InvalidOperationError, IterationSnapshot,
                    MycelError, OptimizerOptions, OutOfMemoryError, PcgResult, StaticAnalysisOptions,
                    StaticAnalysisResult, TimeoutError_, TopologyOptimizationResult)

FP64 = 0
MIXED = 1
FP64_FACTORED = 2
FP64_MG = 3
MIXED_MG = 4
_PREC = {"fp64": FP64, "mixed": MIXED, "fp64f": FP64_FACTORED, "mg": FP64_MG, "mixed-mg": MIXED_MG, FP64: FP64,
         MIXED: MIXED, FP64_FACTORED: FP64_FACTORED, FP64_MG: FP64_MG, MIXED_MG: MIXED_MG}

_ERRORS = {1: ArgumentError, 2: InvalidOperationError, 3: InvalidOperationError, 4: InvalidOperationError,
           5: CancelledError, 6: TimeoutError_, 7: DeviceError, 8: OutOfMemoryError, 9: InvalidOperationError}


def _check(status: int, ctx=None):
    if status == 0:
        return
    lib = L.load()
    msg = lib.mycel_last_error(ctx.handle if ctx is not None else None)
    text = msg.decode("utf-8", "replace") if msg else f"status {status}"
    raise _ERRORS.get(status, MycelError)(text)


class Context:
    """One CUDA device and stream (mycel_ctx)."""

    def __init__(self, device: int = 0):
        lib = L.load()
        h = C.c_void_p()
        _check(lib.mycel_ctx_create(device, C.byref(h)))
        self.handle = h.value
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            L.load().mycel_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return L.load().mycel_ctx_stream(self.handle) or 0

    @property
    def launch_count(self) -> int:
        return int(L.load().mycel_ctx_launch_count(self.handle))

    @property
    def packed_count(self) -> int:
        """Right-hand sides solved through packed launches on this context (mycel_simp_step_many / run_many)."""
        return int(L.load().mycel_ctx_packed_count(self.handle))

    def set_profiling(self, on: bool = True):
        _check(L.load().mycel_ctx_set_profiling(self.handle, int(on)), self)

    def set_oc_wait(self, max_polls: int = 0, unreachable: bool = False):
        """Bounded waits of the OC kernel's grid barrier (0: default); unreachable=True makes every wait run out
        (for testing the MYCEL_E_TIMEOUT path)."""
        _check(L.load().mycel_ctx_set_oc_wait(self.handle, int(max_polls), int(unreachable)), self)

    def kernel_timing(self, which: int = 0) -> dict:
        ms, n, nodes, els = C.c_double(0), C.c_int64(0), C.c_int64(0), C.c_int64(0)
        _check(L.load().mycel_ctx_kernel_timing(self.handle, which, C.byref(ms), C.byref(n), C.byref(nodes),
                                                C.byref(els)), self)
        return dict(total_ms=ms.value, launches=n.value, nodes=nodes.value, active_elements=els.value)


_default_ctx = None
_default_lock = threading.Lock()


def default_context() -> Context:
    global _default_ctx
    with _default_lock:
        if _default_ctx is None:
            _default_ctx = Context(0)
        return _default_ctx


def _pcg_result(r: L.PcgResultC) -> PcgResult:
    msg = r.message.decode("utf-8", "replace")
    return PcgResult(int(r.iterations), float(r.final_residual), bool(r.converged), float(r.elapsed_ms), msg or None,
                     int(r.refinement_steps), int(r.inner_iterations), int(r.fallback_iterations))


class Problem:
    """A FeModel resident on the device (mycel_problem): FeModel + FemOperator state."""

    def __init__(self, model: FeModel, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.model = model
        lib = L.load()
        g = model.grid
        grid = L.Grid(g.nx, g.ny, g.nz, float(np.float32(g.h)))
        mat = L.Material(model.material.e0, model.material.nu, model.material.emin_ratio)
        self._keep = []
        loads = (L.LoadCaseC * max(1, len(model.loads)))()
        for i, lc in enumerate(model.loads):
            nodes = np.ascontiguousarray(lc.patch.nodes, dtype=np.int32)
            areas = np.ascontiguousarray(lc.patch.node_area, dtype=np.float64)
            self._keep += [nodes, areas]
            loads[i].n_nodes = nodes.size
            loads[i].nodes = nodes.ctypes.data
            loads[i].node_area = areas.ctypes.data
            loads[i].force[:] = [np.float32(v) for v in lc.total_force]
        fixed = np.ascontiguousarray(model.fixed_dofs, dtype=np.int32)
        dens = L.f64(model.element_density)
        h = C.c_void_p()
        _check(lib.mycel_problem_create(self.ctx.handle, C.byref(grid), model.domain.ctypes.data, C.byref(mat),
                                        fixed.ctypes.data if fixed.size else None, fixed.size, loads, len(model.loads),
                                        dens.ctypes.data, model.penal, C.byref(h)), self.ctx)
        self.handle = h.value
        self._keep = []

    def close(self):
        if getattr(self, "handle", None):
            for sess in list(getattr(self, "_sessions", ())):
                sess.close()
            L.load().mycel_problem_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- info ----
    def info(self) -> dict:
        pi = L.ProblemInfo()
        _check(L.load().mycel_problem_info_get(self.handle, C.byref(pi)), self.ctx)
        return {k: int(getattr(pi, k)) for k, _ in L.ProblemInfo._fields_}

    @property
    def n_dofs(self) -> int:
        return self.model.total_dofs

    MATVEC32_AUTO, MATVEC32_SIMT, MATVEC32_TENSOR = 0, 1, 2

    def set_matvec32(self, variant: int):
        """FP32 matvec variant of the mixed form: 0 autotune (default), 1 dense KE on the FMA pipe, 2 dense KE on
        the tensor cores, 3 factorised cube-element operator."""
        _check(L.load().mycel_problem_set_tuning(self.handle, 1, int(variant)), self.ctx)

    def kernel_bench(self, which: int, reps: int = 20) -> float:
        """Device microseconds of one launch of a solver kernel (0: FP32 outer matvec, 3: multigrid level-1
        product), from `reps` launches back to back in one CUDA graph timed by CUDA events."""
        us = C.c_double(0)
        _check(L.load().mycel_problem_kernel_bench(self.handle, int(which), int(reps), C.byref(us)), self.ctx)
        return us.value

    def matvec32(self) -> int:
        v = C.c_int32(0)
        _check(L.load().mycel_problem_get_tuning(self.handle, 1, C.byref(v)), self.ctx)
        return v.value

    def forces(self) -> np.ndarray:
        f = np.zeros(self.n_dofs)
        _check(L.load().mycel_problem_forces(self.handle, f.ctypes.data), self.ctx)
        return f

    def load_case_count(self) -> int:
        n = C.c_int32(0)
        _check(L.load().mycel_problem_load_cases(self.handle, C.byref(n)), self.ctx)
        return n.value

    def case_forces(self, k: int) -> np.ndarray:
        """Nodal forces of load case k alone (the right-hand side of case k when load cases are kept apart)."""
        f = np.zeros(self.n_dofs)
        _check(L.load().mycel_problem_case_forces(self.handle, int(k), f.ctypes.data), self.ctx)
        return f

    # ---- FemOperator ----
    def update_densities(self, density_box, penal: float):
        d = L.f64(density_box)
        _check(L.load().mycel_update_densities(self.handle, d.ctypes.data, float(penal)), self.ctx)

    def diagonal(self) -> np.ndarray:
        out = np.zeros(self.n_dofs)
        _check(L.load().mycel_diagonal(self.handle, out.ctypes.data), self.ctx)
        return out

    def apply_k(self, x, projected: bool = False, precision="fp64") -> np.ndarray:
        x = L.f64(x)
        y = np.zeros(self.n_dofs)
        _check(L.load().mycel_apply_k(self.handle, x.ctypes.data, y.ctypes.data, int(projected), _PREC[precision]),
               self.ctx)
        return y

    def apply_a(self, x, precision="fp64") -> np.ndarray:
        return self.apply_k(x, True, precision)

    # ---- PcgSolver ----
    def pcg_solve(self, b, x0=None, tol: float = 1e-6, max_iterations: int = 5000, precision="fp64"):
        b = L.f64(b)
        x = np.zeros(self.n_dofs) if x0 is None else np.array(x0, dtype=np.float64)
        r = L.PcgResultC()
        _check(L.load().mycel_pcg_solve(self.handle, b.ctypes.data, x.ctypes.data, tol, max_iterations,
                                        _PREC[precision], C.byref(r)), self.ctx)
        return x, _pcg_result(r)

    # ---- SensitivityAnalysis ----
    def sensitivities(self, u, rho_phys_active, penal: float) -> np.ndarray:
        u = L.f64(u)
        rho = L.f64(rho_phys_active)
        dc = np.zeros(self.model.active_element_count)
        _check(L.load().mycel_sensitivities(self.handle, u.ctypes.data, rho.ctypes.data, float(penal), dc.ctypes.data),
               self.ctx)
        return dc


class DensityFilter:
    """DensityFilter over a problem's active elements (radius in elements)."""

    def __init__(self, problem: Problem, rmin: float):
        self.problem = problem
        h = C.c_void_p()
        _check(L.load().mycel_filter_create(problem.handle, float(rmin), C.byref(h)), problem.ctx)
        self.handle = h.value
        self.n = problem.model.active_element_count

    def close(self):
        if getattr(self, "handle", None):
            L.load().mycel_filter_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def apply(self, rho_active) -> np.ndarray:
        x = L.f64(rho_active)
        if x.size < self.n:
            raise ArgumentError("Buffer lengths must be at least ActiveCount.")
        out = np.zeros(self.n)
        _check(L.load().mycel_filter_apply(self.handle, x.ctypes.data, out.ctypes.data), self.problem.ctx)
        return out

    def adjoint(self, dc_active) -> np.ndarray:
        x = L.f64(dc_active)
        if x.size < self.n:
            raise ArgumentError("Buffer lengths must be at least ActiveCount.")
        out = np.zeros(self.n)
        _check(L.load().mycel_filter_adjoint(self.handle, x.ctypes.data, out.ctypes.data), self.problem.ctx)
        return out

    @property
    def s(self) -> np.ndarray:
        out = np.zeros(self.n)
        _check(L.load().mycel_filter_s(self.handle, out.ctypes.data), self.problem.ctx)
        return out


def oc_update(rho, dc, s, passive, target_volume_fraction, move_limit=0.2, rho_min=1e-3, lambda_guess=1.0,
              max_bisection_steps=60, volume_tolerance=1e-8, ctx: Optional[Context] = None):
    """OcOptimizer.Update; returns (rho_new, lambda)."""
    ctx = ctx or default_context()
    rho = L.f64(rho)
    n = rho.size
    dc = L.f64(dc)
    s = L.f64(s)
    if dc.size < n or s.size < n:
        raise ArgumentError("All spans must have length >= rho.Length.")
    pas = None if passive is None else np.ascontiguousarray(passive, dtype=np.uint8)
    out = np.zeros(n)
    lam = C.c_double(0)
    _check(L.load().mycel_oc_update(ctx.handle, n, rho.ctypes.data, dc.ctypes.data, s.ctypes.data, L.ptr(pas),
                                    out.ctypes.data, target_volume_fraction, move_limit, rho_min, lambda_guess,
                                    max_bisection_steps, volume_tolerance, C.byref(lam)), ctx)
    return out, lam.value


class HeavisideProjection:
    """HeavisideProjection.Project / Derivative (HeavisideProjection.cs:12-37) on the device."""

    @staticmethod
    def project(rho_tilde, beta: float, eta: float = 0.5, ctx: Optional[Context] = None) -> np.ndarray:
        ctx = ctx or default_context()
        x = L.f64(rho_tilde).ravel()
        out = np.empty(x.size)
        _check(L.load().mycel_heaviside_project(ctx.handle, x.size, x.ctypes.data, out.ctypes.data, beta, eta), ctx)
        return out

    @staticmethod
    def derivative(rho_tilde, beta: float, eta: float = 0.5, ctx: Optional[Context] = None) -> np.ndarray:
        ctx = ctx or default_context()
        x = L.f64(rho_tilde).ravel()
        out = np.empty(x.size)
        _check(L.load().mycel_heaviside_derivative(ctx.handle, x.size, x.ctypes.data, out.ctypes.data, beta, eta),
               ctx)
        return out


def math_pow(x, y, ctx: Optional[Context] = None) -> np.ndarray:
    """Math.Pow as the kernels evaluate it on the device (the host C library's pow, bit for bit):
    x**y elementwise, y an array of x's length or a scalar."""
    ctx = ctx or default_context()
    x = L.f64(x).ravel()
    y = L.f64(np.atleast_1d(y)).ravel()
    out = np.empty(x.size)
    _check(L.load().mycel_pow(ctx.handle, x.size, x.ctypes.data, y.ctypes.data, y.size, out.ctypes.data), ctx)
    return out


class StaticAnalysis:
    @staticmethod
    def run(model: FeModel, options: Optional[StaticAnalysisOptions] = None, ctx: Optional[Context] = None,
            reactions: bool = True, von_mises: bool = True) -> StaticAnalysisResult:
        options = options or StaticAnalysisOptions()
        prob = Problem(model, ctx)
        try:
            n = model.total_dofs
            u = np.zeros(n)
            rx = np.zeros(n) if reactions else None
            vm = np.zeros(model.total_elements) if von_mises else None
            ws = None if options.warm_start_displacements is None else L.f64(options.warm_start_displacements)
            o = L.StaticOptions(options.tolerance, options.max_iterations, int(options.throw_on_non_convergence),
                                _PREC[options.precision])
            c = C.c_double(0)
            md = C.c_double(0)
            r = L.PcgResultC()
            _check(L.load().mycel_static_solve(prob.handle, C.byref(o), L.ptr(ws), 0 if ws is None else ws.size,
                                               u.ctypes.data, L.ptr(rx), L.ptr(vm), C.byref(c), C.byref(md),
                                               C.byref(r)), prob.ctx)
            return StaticAnalysisResult(u, c.value, rx, md.value, _pcg_result(r), vm)
        finally:
            prob.close()

    @staticmethod
    def run_cases(model: FeModel, options: Optional[StaticAnalysisOptions] = None,
                  ctx: Optional[Context] = None) -> List[StaticAnalysisResult]:
        """StaticAnalysis.Run for every load case apart on one stiffness (multi-RHS; the reference sums its load
        cases). Case k equals StaticAnalysis.Run on the model holding case k alone; E, DiagA and the solver's
        set-up are formed once. Each case starts from zero; reactions and von Mises are not formed."""
        options = options or StaticAnalysisOptions()
        prob = Problem(model, ctx)
        try:
            m = prob.load_case_count()
            n = model.total_dofs
            u = np.zeros((m, n))
            c = np.zeros(m)
            md = np.zeros(m)
            rs = (L.PcgResultC * max(m, 1))()
            o = L.StaticOptions(options.tolerance, options.max_iterations, int(options.throw_on_non_convergence),
                                _PREC[options.precision])
            _check(L.load().mycel_static_solve_cases(prob.handle, C.byref(o), u.ctypes.data, c.ctypes.data,
                                                     md.ctypes.data, rs), prob.ctx)
            return [StaticAnalysisResult(u[k], float(c[k]), None, float(md[k]), _pcg_result(rs[k]), None)
                    for k in range(m)]
        finally:
            prob.close()

    @staticmethod
    def average_element_to_node(model: FeModel, element_scalar, ctx: Optional[Context] = None,
                                problem: Optional["Problem"] = None) -> np.ndarray:
        """StaticAnalysis.AverageElementToNode: nodal means of an element scalar over the active elements."""
        prob = problem or Problem(model, ctx)
        try:
            es = np.ascontiguousarray(element_scalar, dtype=np.float64).reshape(-1)
            out = np.zeros(model.total_nodes)
            _check(L.load().mycel_average_element_to_node(prob.handle, es.ctypes.data, es.size, out.ctypes.data),
                   prob.ctx)
            return out
        finally:
            if problem is None:
                prob.close()


class IterationController:
    """Cooperative pause / resume / stop between SIMP iterations (IterationController.cs:9-65)."""

    def __init__(self):
        self._cancel = C.c_int32(0)
        self._pause = C.c_int32(0)

    def pause(self):
        self._pause.value = 1

    def resume(self):
        self._pause.value = 0

    def stop(self):
        self._cancel.value = 1
        self._pause.value = 0

    def reset(self):
        self._cancel.value = 0
        self._pause.value = 0

    @property
    def is_paused(self):
        return bool(self._pause.value)

    @property
    def is_stopped(self):
        return bool(self._cancel.value)


def _simp_options(o: OptimizerOptions, keep: list) -> L.SimpOptions:
    def arr(a, dt):
        if a is None:
            return None, 0
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data, a.size

    pm, pl = arr(o.passive_mask, np.uint8)
    idp, idl = arr(o.initial_density, np.float32)
    wp, wl = arr(o.warm_start_displacements, np.float64)
    return L.SimpOptions(o.volume_fraction, o.filter_radius_mm, o.penal, o.move_limit, o.max_iterations,
                         o.solver_tolerance_initial, o.solver_tolerance_final, o.solver_max_iterations,
                         int(o.continuation), int(o.enable_heaviside), o.rho_min, pm, pl,
                         int(o.protect_boundary_hinges), idp, idl, o.start_iteration, wp, wl,
                         int(o.enforce_minimum_filter_radius), _PREC[o.precision], int(o.separate_load_cases))


def _snapshot(r: L.IterRecord, phys=None, design=None) -> IterationSnapshot:
    return IterationSnapshot(int(r.iteration), r.compliance, r.volume_fraction, r.max_change, r.grey_level,
                             int(r.solver_iterations), r.solver_residual, r.max_displacement, r.solve_ms,
                             r.sensitivity_ms, r.filter_ms, r.update_ms, r.total_ms, phys, design)


class TopologyOptimizer:
    @staticmethod
    def run_many(models: Sequence[FeModel], options=None, ctx: Optional[Context] = None,
                 controller: Optional[IterationController] = None) -> List[TopologyOptimizationResult]:
        """Several optimisations side by side on one GPU, one SIMP iteration of each per step
        (mycel_simp_step_many): the mixed multigrid form's solves are packed into shared launches. options is
        one OptimizerOptions for all or one per model. Each result equals TopologyOptimizer.run's for that
        model alone with the same options; the snapshots carry densities only for the last iteration."""
        if isinstance(options, OptimizerOptions) or options is None:
            options = [options or OptimizerOptions()] * len(models)
        return _run_many(list(models), list(options), ctx, controller)

    @staticmethod
    def run(model: FeModel, options: Optional[OptimizerOptions] = None,
            progress: Optional[Callable[[IterationSnapshot], None]] = None,
            controller: Optional[IterationController] = None, ctx: Optional[Context] = None,
            keep_snapshots: bool = False) -> TopologyOptimizationResult:
        options = options or OptimizerOptions()
        prob = Problem(model, ctx)
        keep = []
        try:
            so = _simp_options(options, keep)
            cap = max(1, options.max_iterations - options.start_iteration + 1)
            hist = (L.IterRecord * cap)()
            ni = C.c_int32(0)
            cv = C.c_int32(0)
            u = np.zeros(model.total_dofs)
            phys = np.zeros(model.total_elements, dtype=np.float32)
            des = np.zeros(model.total_elements, dtype=np.float32)
            snaps_arrays = {}
            ne = model.total_elements

            def cb(user, rec, pp, dp):
                r = rec.contents
                pa = np.ctypeslib.as_array(pp, shape=(ne,)).copy() if (keep_snapshots or progress) else None
                da = np.ctypeslib.as_array(dp, shape=(ne,)).copy() if (keep_snapshots or progress) else None
                if keep_snapshots:
                    snaps_arrays[int(r.iteration)] = (pa, da)
                if progress is not None:
                    progress(_snapshot(r, pa, da))

            cfn = L.PROGRESS_FN(cb) if (progress is not None or keep_snapshots) else L.PROGRESS_FN()
            cancel = controller._cancel if controller else None
            pause = controller._pause if controller else None
            st = L.load().mycel_simp_run(prob.handle, C.byref(so), cfn, None,
                                         C.addressof(cancel) if cancel is not None else None,
                                         C.addressof(pause) if pause is not None else None, hist, cap, C.byref(ni),
                                         C.byref(cv), u.ctypes.data, phys.ctypes.data, des.ctypes.data)
            _check(st, prob.ctx)
            snaps = []
            for r in hist[:ni.value]:
                pa, da = snaps_arrays.get(int(r.iteration), (None, None))
                snaps.append(_snapshot(r, pa, da))
            if snaps:
                snaps[-1].physical_density = phys
                snaps[-1].design_density = des
            final_c = snaps[-1].compliance if snaps else 0.0
            final_v = snaps[-1].volume_fraction if snaps else 0.0
            return TopologyOptimizationResult(bool(cv.value), ni.value, snaps, final_c, final_v, phys, des, u)
        finally:
            prob.close()


def _run_many(models: Sequence[FeModel], options: Sequence[OptimizerOptions], ctx: Optional["Context"] = None,
              controller: Optional[IterationController] = None) -> List[TopologyOptimizationResult]:
    ctx = ctx or default_context()
    probs = []
    sess = []
    try:
        probs = [Problem(m, ctx) for m in models]
        sess = [SimpSession(p, o) for p, o in zip(probs, options)]
        snaps = SimpSession.run_many(sess, controller)
        res = []
        for s, sn in zip(sess, snaps):
            d = s.read(u=True, densities=True)
            if sn:
                sn[-1].physical_density = d["physical"]
                sn[-1].design_density = d["design"]
            res.append(TopologyOptimizationResult(s.converged, len(sn), sn, sn[-1].compliance if sn else 0.0,
                                                  sn[-1].volume_fraction if sn else 0.0, d["physical"], d["design"],
                                                  d["u"]))
        return res
    finally:
        for s in sess:
            s.close()
        for p in probs:
            p.close()


class SimpSession:
    """Device-resident SIMP state stepped by the caller (mycel_simp_begin / step / read / end)."""

    def __init__(self, problem: Problem, options: OptimizerOptions):
        self.problem = problem
        self._keep = []
        so = _simp_options(options, self._keep)
        h = C.c_void_p()
        _check(L.load().mycel_simp_begin(problem.handle, C.byref(so), C.byref(h)), problem.ctx)
        self.handle = h.value
        self.done = False
        self._max_iterations = max(1, int(options.max_iterations) - int(options.start_iteration) + 1)
        if not hasattr(problem, "_sessions"):
            problem._sessions = weakref.WeakSet()
        problem._sessions.add(self)

    def step(self) -> IterationSnapshot:
        r = L.IterRecord()
        d = C.c_int32(0)
        _check(L.load().mycel_simp_step(self.handle, C.byref(r), C.byref(d)), self.problem.ctx)
        self.done = bool(d.value)
        return _snapshot(r)

    @staticmethod
    def step_many(sessions: Sequence["SimpSession"], controller: Optional[IterationController] = None):
        """One SIMP iteration of each session (mycel_simp_step_many): one context, one session per problem.
        Sessions in the mixed multigrid form have their solves packed (one launch per kernel of an outer
        iteration for all of them); each takes the iteration its own step() would take. Returns the
        snapshots (None for a session that was done already)."""
        n = len(sessions)
        if n == 0:
            return []
        hs = (C.c_void_p * n)(*[s.handle for s in sessions])
        recs = (L.IterRecord * n)()
        done = (C.c_int32 * n)()
        stat = (C.c_int32 * n)()
        was_done = [s.done for s in sessions]
        cancel = controller._cancel if controller else None
        st = L.load().mycel_simp_step_many(hs, n, recs, done, stat,
                                           C.addressof(cancel) if cancel is not None else None)
        for k, s in enumerate(sessions):
            if stat[k] == 0:
                s.done = bool(done[k])
        _check(st, sessions[0].problem.ctx)
        return [None if was_done[k] else _snapshot(recs[k]) for k in range(n)]

    @staticmethod
    def run_many(sessions: Sequence["SimpSession"], controller: Optional[IterationController] = None, cap: int = 0):
        """Every session to its end (mycel_simp_run_many): one context, one session per problem. In the mixed
        multigrid form the solves share one packed plan and each problem goes on to its next SIMP iteration as
        soon as its own solve ends. Returns each session's snapshots (records only)."""
        n = len(sessions)
        if n == 0:
            return []
        cap = cap or max(1, max(s._max_iterations for s in sessions))
        hs = (C.c_void_p * n)(*[s.handle for s in sessions])
        hist = (L.IterRecord * (n * cap))()
        nit = (C.c_int32 * n)()
        stat = (C.c_int32 * n)()
        cancel = controller._cancel if controller else None
        st = L.load().mycel_simp_run_many(hs, n, hist, cap, nit, stat,
                                          C.addressof(cancel) if cancel is not None else None)
        out = [[_snapshot(hist[k * cap + q]) for q in range(min(nit[k], cap))] for k in range(n)]
        stopped = cancel is not None and bool(cancel.value)
        for s in sessions:
            s.done = s.done or not stopped
        _check(st, sessions[0].problem.ctx)
        return out

    @property
    def converged(self) -> bool:
        """The stop rule has fired (TopologyOptimizationResult.Converged)."""
        return bool(L.load().mycel_simp_converged(self.handle))

    def read(self, u=True, densities=True, active=False, out: Optional[dict] = None):
        """u, the physical and design densities (box, float) and, with active, the active-indexed FP64
        densities. out may hold preallocated arrays ("u", "physical", "design"; pinned host memory makes the
        copies faster), which are filled and returned instead of new ones."""
        m = self.problem.model
        out = out or {}

        def buf(key, want, n, dt):
            if not want:
                return None
            a = out.get(key)
            if a is None:
                return np.zeros(n, dtype=dt)
            if a.dtype != np.dtype(dt) or a.size != n or not a.flags.c_contiguous:
                raise ArgumentError(f"out[{key!r}]: {n} contiguous {np.dtype(dt).name} values expected")
            return a
        uu = buf("u", u, m.total_dofs, np.float64)
        ph = buf("physical", densities, m.total_elements, np.float32)
        de = buf("design", densities, m.total_elements, np.float32)
        rpa = np.zeros(m.active_element_count) if active else None
        rda = np.zeros(m.active_element_count) if active else None
        lam = C.c_double(0)
        _check(L.load().mycel_simp_read(self.handle, L.ptr(uu), L.ptr(ph), L.ptr(de), L.ptr(rpa), L.ptr(rda),
                                        C.byref(lam)), self.problem.ctx)
        return dict(u=uu, physical=ph, design=de, rho_phys_active=rpa, rho_design_active=rda, lam=lam.value)

    def surface_mesh(self, threshold: float = 0.5, origin=(0.0, 0.0, 0.0)):
        """Iso-surface (SurfaceNetsExtractor.Extract) of the last iteration's physical density, extracted from
        the device-resident field (no host copy of the density)."""
        o = np.ascontiguousarray(origin, dtype=np.float32)
        lib = L.load()
        h = C.c_void_p()
        _check(lib.mycel_simp_surface_nets(self.handle, o.ctypes.data, float(threshold), C.byref(h)), self.problem.ctx)
        try:
            nv, ni, passes, changes = C.c_int64(0), C.c_int64(0), C.c_int32(0), C.c_int64(0)
            _check(lib.mycel_mesh_info(h, C.byref(nv), C.byref(ni), C.byref(passes), C.byref(changes)))
            pos = np.zeros((nv.value, 3), dtype=np.float32)
            idx = np.zeros(ni.value, dtype=np.int32)
            _check(lib.mycel_mesh_copy(h, pos.ctypes.data, idx.ctypes.data))
        finally:
            lib.mycel_mesh_destroy(h)
        return IndexedMesh(pos, idx, int(passes.value), int(changes.value))

    def frame_begin(self) -> int:
        """Start the RunWriter frame of the last iteration (quantised on the device, copied without waiting)."""
        slot = C.c_int32(-1)
        _check(L.load().mycel_simp_frame_begin(self.handle, C.byref(slot)), self.problem.ctx)
        return slot.value

    def frame_end(self, slot: int):
        """(frame bytes [box], 72-byte header, FNV-1a checksum) of a frame started by frame_begin."""
        m = self.problem.model
        fr = np.zeros(m.total_elements, dtype=np.uint8)
        hd = np.zeros(72, dtype=np.uint8)
        ck = C.c_uint32(0)
        _check(L.load().mycel_simp_frame_end(self.handle, slot, fr.ctypes.data, hd.ctypes.data, C.byref(ck)),
               self.problem.ctx)
        return fr, bytes(hd), ck.value

    def close(self):
        if getattr(self, "handle", None):
            if getattr(self.problem, "handle", None):  # a destroyed problem has ended its sessions already
                L.load().mycel_simp_end(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _server_check(status: int, handle):
    if status == 0:
        return
    msg = L.load().mycel_server_last_error(handle)
    text = msg.decode("utf-8", "replace") if msg else f"status {status}"
    raise _ERRORS.get(status, MycelError)(text)


_JOB_STATES = {0: "queued", 1: "running", 2: "done", 3: "failed"}


class Server:
    """Continuous batching of SIMP jobs on one GPU (mycel_server): ``slots`` jobs run at once on their own
    streams, admitted in arrival order (with backfill) against ``hbm_budget_bytes`` of device memory."""

    def __init__(self, slots: int = 4, hbm_budget_bytes: int = 150 * 10**9, device: int = 0):
        so = L.ServerOptions(device, slots, int(hbm_budget_bytes))
        h = C.c_void_p()
        st = L.load().mycel_server_create(C.byref(so), C.byref(h))
        if st:
            _check(st, None)
        self.handle = h.value
        self._models = {}

    @staticmethod
    def _spec(model: FeModel, options: OptimizerOptions, keep_u: bool, keep: list) -> L.JobSpec:
        g = model.grid
        loads = (L.LoadCaseC * max(1, len(model.loads)))()
        for i, lc in enumerate(model.loads):
            nodes = np.ascontiguousarray(lc.patch.nodes, dtype=np.int32)
            areas = np.ascontiguousarray(lc.patch.node_area, dtype=np.float64)
            keep += [nodes, areas]
            loads[i].n_nodes = nodes.size
            loads[i].nodes = nodes.ctypes.data
            loads[i].node_area = areas.ctypes.data
            loads[i].force[:] = [np.float32(v) for v in lc.total_force]
        fixed = np.ascontiguousarray(model.fixed_dofs, dtype=np.int32)
        dom = np.ascontiguousarray(model.domain, dtype=np.uint8)
        dens = L.f64(model.element_density)
        keep += [loads, fixed, dom, dens]
        return L.JobSpec(L.Grid(g.nx, g.ny, g.nz, float(np.float32(g.h))), dom.ctypes.data,
                         L.Material(model.material.e0, model.material.nu, model.material.emin_ratio),
                         fixed.ctypes.data if fixed.size else None, fixed.size, C.cast(loads, C.c_void_p),
                         len(model.loads), dens.ctypes.data, model.penal, _simp_options(options, keep),
                         int(bool(keep_u)))

    @staticmethod
    def device_bytes(model: FeModel, options: OptimizerOptions) -> int:
        """Admission estimate of one job (mycel_job_device_bytes)."""
        keep = []
        spec = Server._spec(model, options, False, keep)
        return int(L.load().mycel_job_device_bytes(C.byref(spec)))

    def submit(self, model: FeModel, options: OptimizerOptions, keep_u: bool = False) -> int:
        keep = []
        spec = self._spec(model, options, keep_u, keep)
        jid = C.c_int64(-1)
        _server_check(L.load().mycel_server_submit(self.handle, C.byref(spec), C.byref(jid)), self.handle)
        self._models[jid.value] = model
        return jid.value

    def info(self, job: int) -> dict:
        ji = L.JobInfo()
        _server_check(L.load().mycel_server_job_info(self.handle, job, C.byref(ji)), self.handle)
        d = {k: getattr(ji, k) for k, _ in L.JobInfo._fields_}
        d["message"] = ji.message.decode("utf-8", "replace")
        d["state"] = _JOB_STATES.get(ji.state, str(ji.state))
        return d

    def wait(self, job: int = -1, timeout: Optional[float] = None) -> None:
        _server_check(L.load().mycel_server_wait(self.handle, job, -1.0 if timeout is None else float(timeout)),
                      self.handle)

    def result(self, job: int, u: bool = False) -> dict:
        m = self._models[job]
        info = self.info(job)
        cap = max(1, int(info["iterations"]))
        hist = (L.IterRecord * cap)()
        ph = np.zeros(m.total_elements, dtype=np.float32)
        de = np.zeros(m.total_elements, dtype=np.float32)
        uu = np.zeros(m.total_dofs) if u else None
        _server_check(L.load().mycel_server_job_result(self.handle, job, hist, cap, ph.ctypes.data, de.ctypes.data,
                                                       L.ptr(uu)), self.handle)
        return dict(info=info, history=[_snapshot(r) for r in hist[:info["iterations"]]], physical=ph, design=de,
                    u=uu)

    def stats(self) -> dict:
        s = L.ServerStats()
        _server_check(L.load().mycel_server_stats_get(self.handle, C.byref(s)), self.handle)
        return {k: getattr(s, k) for k, _ in L.ServerStats._fields_}

    def close(self):
        if getattr(self, "handle", None):
            L.load().mycel_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class IndexedMesh:
    """Triangle mesh (Geometry/IndexedMesh.cs): positions [V, 3] float32, indices [3T] int32 (counter-clockwise
    seen from outside), plus the well-composedness passes and resolutions of the extraction."""
    positions: np.ndarray
    indices: np.ndarray
    passes: int = 0
    changes: int = 0

    @property
    def vertex_count(self) -> int:
        return int(self.positions.shape[0])

    @property
    def triangle_count(self) -> int:
        return int(self.indices.size // 3)


class SurfaceNetsExtractor:
    """SurfaceNetsExtractor.Extract (PostProcessing/SurfaceNetsExtractor.cs:31-312) on the device."""

    @staticmethod
    def extract(grid, physical_density, threshold: float = 0.5, ctx: Context = None) -> IndexedMesh:
        ctx = ctx or default_context()
        d = np.ascontiguousarray(physical_density, dtype=np.float32).reshape(-1)
        o = np.ascontiguousarray(getattr(grid, "origin", (0.0, 0.0, 0.0)), dtype=np.float32)
        lib = L.load()
        h = C.c_void_p()
        _check(lib.mycel_surface_nets(ctx.handle, grid.nx, grid.ny, grid.nz, float(grid.h), o.ctypes.data,
                                      d.ctypes.data, d.size, float(threshold), C.byref(h)), ctx)
        try:
            nv, ni, passes, changes = C.c_int64(0), C.c_int64(0), C.c_int32(0), C.c_int64(0)
            _check(lib.mycel_mesh_info(h, C.byref(nv), C.byref(ni), C.byref(passes), C.byref(changes)))
            pos = np.zeros((nv.value, 3), dtype=np.float32)
            idx = np.zeros(ni.value, dtype=np.int32)
            _check(lib.mycel_mesh_copy(h, pos.ctypes.data, idx.ctypes.data))
        finally:
            lib.mycel_mesh_destroy(h)
        return IndexedMesh(pos, idx, int(passes.value), int(changes.value))


class TaubinSmoother:
    """TaubinSmoother.Smooth (PostProcessing/TaubinSmoother.cs:15-134) on the device."""

    @staticmethod
    def smooth(mesh: IndexedMesh, iterations: int = 3, lam: float = 0.50, mu: float = -0.53,
               ctx: Context = None) -> IndexedMesh:
        ctx = ctx or default_context()
        pos = np.array(mesh.positions, dtype=np.float32, copy=True, order="C")
        idx = np.ascontiguousarray(mesh.indices, dtype=np.int32)
        _check(L.load().mycel_taubin_smooth(ctx.handle, pos.ctypes.data, pos.shape[0], idx.ctypes.data, idx.size,
                                            int(iterations), float(lam), float(mu)), ctx)
        return IndexedMesh(pos, idx.copy(), mesh.passes, mesh.changes)
