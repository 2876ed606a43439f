"""ORACLE — test infrastructure only.

ctypes wrapper of the CPU restatement in oracle.cpp (see oracle.h for what it restates and how it is pinned).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

from mycel_b200.model import (ArgumentError, FeModel, InvalidOperationError, OptimizerOptions, PcgResult,
                              StaticAnalysisResult)

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def _load():
    if not os.path.exists(_LIB):
        build()
    return C.CDLL(_LIB)


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
        _setup(_lib)
    return _lib


P = C.c_void_p
dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
fp = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
bp = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


class PcgRes(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("final_residual", C.c_double), ("converged", C.c_int32),
                ("message", C.c_char * 256)]


class SimpOpts(C.Structure):
    _fields_ = [("volume_fraction", C.c_double), ("filter_radius_mm", C.c_double), ("penal", C.c_double),
                ("move_limit", C.c_double), ("max_iterations", C.c_int32), ("solver_tol_initial", C.c_double),
                ("solver_tol_final", C.c_double), ("solver_max_iterations", C.c_int32), ("continuation", C.c_int32),
                ("enable_heaviside", C.c_int32), ("rho_min", C.c_double), ("passive_mask", P),
                ("passive_len", C.c_int64), ("protect_boundary_hinges", C.c_int32), ("initial_density", P),
                ("initial_density_len", C.c_int64), ("start_iteration", C.c_int32), ("warm_start", P),
                ("warm_start_len", C.c_int64), ("enforce_min_filter_radius", C.c_int32),
                ("separate_load_cases", C.c_int32)]


class IterRec(C.Structure):
    _fields_ = [("iteration", C.c_int32), ("compliance", C.c_double), ("volume_fraction", C.c_double),
                ("max_change", C.c_double), ("grey_level", C.c_double), ("solver_iterations", C.c_int32),
                ("solver_residual", C.c_double), ("max_displacement", C.c_double), ("total_ms", C.c_double)]


def _setup(L):
    L.orc_quantized_checksum.restype = C.c_uint32
    L.orc_quantized_checksum.argtypes = [np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS"), C.c_int64, P]
    L.orc_create_ke.argtypes = [C.c_double, C.c_double, dp]
    L.orc_model_create.restype = P
    L.orc_model_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, bp, C.c_double, C.c_double, C.c_double, ip,
                                   C.c_int32, P, C.c_double, C.POINTER(C.c_int), C.c_char_p, C.c_int]
    L.orc_model_add_load.argtypes = [P, C.c_int32, ip, dp, C.c_float, C.c_float, C.c_float]
    L.orc_model_free.argtypes = [P]
    L.orc_model_counts.argtypes = [P, np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")]
    L.orc_model_active_elements.argtypes = [P, ip]
    L.orc_model_constrained.argtypes = [P, bp]
    L.orc_model_assemble_forces.argtypes = [P, dp, C.c_char_p, C.c_int]
    L.orc_model_assemble_case_forces.argtypes = [P, C.c_int32, dp, C.c_char_p, C.c_int]
    L.orc_model_load_case_count.restype = C.c_int32
    L.orc_model_load_case_count.argtypes = [P]
    L.orc_model_set_density.argtypes = [P, dp, C.c_double]
    L.orc_op_create.restype = P
    L.orc_op_create.argtypes = [P]
    L.orc_op_free.argtypes = [P]
    L.orc_op_update_densities.argtypes = [P, dp, C.c_double]
    L.orc_op_diag.argtypes = [P, dp]
    L.orc_op_apply_k.argtypes = [P, dp, dp]
    L.orc_op_apply_k_scalar_reference.argtypes = [P, dp, dp]
    L.orc_op_apply_a.argtypes = [P, dp, dp, C.c_int]
    L.orc_op_element_e.argtypes = [P, dp]
    L.orc_pcg_solve.argtypes = [P, dp, dp, C.c_double, C.c_int32, C.POINTER(PcgRes), C.c_char_p, C.c_int]
    L.orc_static_run.argtypes = [P, C.c_double, C.c_int32, P, C.c_int64, C.c_int, dp, P, C.POINTER(C.c_double),
                                 C.POINTER(C.c_double), C.POINTER(PcgRes), C.c_char_p, C.c_int]
    L.orc_von_mises.argtypes = [P, dp, dp]
    L.orc_filter_create.restype = P
    L.orc_filter_create.argtypes = [C.c_int, C.c_int, C.c_int, bp, ip, C.c_int32, C.c_double]
    L.orc_filter_free.argtypes = [P]
    L.orc_filter_apply.argtypes = [P, dp, dp]
    L.orc_filter_adjoint.argtypes = [P, dp, dp]
    L.orc_filter_s.argtypes = [P, dp]
    L.orc_filter_nnz.restype = C.c_int64
    L.orc_filter_nnz.argtypes = [P]
    L.orc_sensitivities.argtypes = [P, dp, dp, dp, C.c_double]
    L.orc_oc_update.restype = C.c_double
    L.orc_oc_update.argtypes = [dp, dp, dp, P, dp, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double,
                                C.c_int32, C.c_double]
    L.orc_oc_trace.restype = C.c_int32
    L.orc_oc_trace.argtypes = [dp, dp, dp, P, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32,
                               C.c_double, dp, dp, C.c_int32, C.POINTER(C.c_double)]
    L.orc_heaviside_project.argtypes = [dp, dp, C.c_int32, C.c_double, C.c_double]
    L.orc_heaviside_derivative.argtypes = [dp, dp, C.c_int32, C.c_double, C.c_double]
    L.orc_passive_region.argtypes = [C.c_int, C.c_int, C.c_int, ip, C.c_int32, C.c_int, bp]
    L.orc_topopt_run.argtypes = [P, C.POINTER(SimpOpts), C.POINTER(IterRec), C.c_int32, C.POINTER(C.c_int32),
                                 C.POINTER(C.c_int32), dp, fp, fp, dp, dp, C.POINTER(C.c_double), C.c_char_p, C.c_int]
    L.orc_set_lane_mode.argtypes = [C.c_int]
    L.orc_math_pow.argtypes = [C.c_int64, dp, dp, C.c_int64, dp]
    L.orc_set_threads.argtypes = [C.c_int]
    L.orc_get_threads.restype = C.c_int


def set_modes(lane_mode: int = 0, threads: int | None = None):
    L = lib()
    L.orc_set_lane_mode(lane_mode)
    if threads is not None:
        L.orc_set_threads(threads)


def math_pow(x, y) -> np.ndarray:
    """Math.Pow as the restatement evaluates it (the C library's pow), elementwise; y an array or a scalar."""
    x = np.ascontiguousarray(x, dtype=np.float64).ravel()
    y = np.ascontiguousarray(np.atleast_1d(y), dtype=np.float64).ravel()
    if y.size not in (1, x.size):
        raise ValueError("y needs 1 or len(x) values")
    out = np.empty(x.size)
    lib().orc_math_pow(x.size, x, y, y.size, out)
    return out


def create_ke(h: float, nu: float) -> np.ndarray:
    ke = np.zeros(576)
    if lib().orc_create_ke(h, nu, ke) != 0:
        raise ArgumentError("Element edge length h must be positive.")
    return ke.reshape(24, 24)


def _raise(st, msg):
    text = msg.value.decode("utf-8", "replace")
    if st == 1:
        raise ArgumentError(text)
    raise InvalidOperationError(text)


class Model:
    """Oracle FeModel (+ FemOperator) built from a mycel_b200.model.FeModel."""

    def __init__(self, fe: FeModel):
        L = lib()
        self.fe = fe
        g = fe.grid
        st = C.c_int(0)
        msg = C.create_string_buffer(512)
        dens = np.ascontiguousarray(fe.element_density, dtype=np.float64)
        self.h = L.orc_model_create(g.nx, g.ny, g.nz, float(np.float32(g.h)), fe.domain, fe.material.e0,
                                    fe.material.nu, fe.material.emin_ratio, fe.fixed_dofs, fe.fixed_dofs.size,
                                    dens.ctypes.data, fe.penal, C.byref(st), msg, 512)
        if not self.h:
            _raise(st.value, msg)
        for lc in fe.loads:
            L.orc_model_add_load(self.h, lc.patch.node_count, lc.patch.nodes, lc.patch.node_area, *lc.total_force)
        self._op = None

    def __del__(self):
        try:
            if self._op:
                lib().orc_op_free(self._op)
            if self.h:
                lib().orc_model_free(self.h)
        except Exception:
            pass

    @property
    def op(self):
        if self._op is None:
            self._op = lib().orc_op_create(self.h)
        return self._op

    def counts(self):
        o = np.zeros(6, dtype=np.int64)
        lib().orc_model_counts(self.h, o)
        return dict(active_elements=int(o[0]), active_nodes=int(o[1]), active_fixed=int(o[2]), dofs=int(o[3]),
                    elements=int(o[4]), nodes=int(o[5]))

    def average_element_to_node(self, element_scalar):
        """StaticAnalysis.AverageElementToNode."""
        es = np.ascontiguousarray(element_scalar, dtype=np.float64)
        out = np.zeros(self.fe.total_nodes)
        L = lib()
        L.orc_average_element_to_node.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_average_element_to_node(self.h, es.ctypes.data, out.ctypes.data)
        return out

    def constrained(self):
        out = np.zeros(self.fe.total_dofs, dtype=np.uint8)
        lib().orc_model_constrained(self.h, out)
        return out

    def active_elements(self):
        out = np.zeros(self.counts()["active_elements"], dtype=np.int32)
        lib().orc_model_active_elements(self.h, out)
        return out

    def forces(self):
        f = np.zeros(self.fe.total_dofs)
        msg = C.create_string_buffer(512)
        st = lib().orc_model_assemble_forces(self.h, f, msg, 512)
        if st:
            _raise(st, msg)
        return f

    def case_forces(self, k):
        """Load case k alone (the right-hand side of case k when load cases are kept separate)."""
        f = np.zeros(self.fe.total_dofs)
        msg = C.create_string_buffer(512)
        st = lib().orc_model_assemble_case_forces(self.h, int(k), f, msg, 512)
        if st:
            _raise(st, msg)
        return f

    def load_case_count(self):
        return int(lib().orc_model_load_case_count(self.h))

    def update_densities(self, dens_box, penal):
        lib().orc_op_update_densities(self.op, np.ascontiguousarray(dens_box, dtype=np.float64), float(penal))

    def diag(self):
        out = np.zeros(self.fe.total_dofs)
        lib().orc_op_diag(self.op, out)
        return out

    def element_e(self):
        out = np.zeros(self.fe.total_elements)
        lib().orc_op_element_e(self.op, out)
        return out

    def apply_k(self, x):
        y = np.zeros(self.fe.total_dofs)
        lib().orc_op_apply_k(self.op, np.ascontiguousarray(x, dtype=np.float64), y)
        return y

    def apply_k_scalar_reference(self, x):
        y = np.zeros(self.fe.total_dofs)
        lib().orc_op_apply_k_scalar_reference(self.op, np.ascontiguousarray(x, dtype=np.float64), y)
        return y

    def apply_a(self, x, projected=True):
        y = np.zeros(self.fe.total_dofs)
        lib().orc_op_apply_a(self.op, np.ascontiguousarray(x, dtype=np.float64), y, int(projected))
        return y

    def pcg_solve(self, b, x0=None, tol=1e-6, max_iter=5000):
        x = np.zeros(self.fe.total_dofs) if x0 is None else np.array(x0, dtype=np.float64)
        r = PcgRes()
        msg = C.create_string_buffer(512)
        st = lib().orc_pcg_solve(self.op, np.ascontiguousarray(b, dtype=np.float64), x, tol, max_iter, C.byref(r),
                                 msg, 512)
        if st:
            _raise(st, msg)
        return x, PcgResult(r.iterations, r.final_residual, bool(r.converged), 0.0, r.message.decode() or None)

    def sensitivities(self, u, rho_phys_active, penal):
        dc = np.zeros(self.counts()["active_elements"])
        lib().orc_sensitivities(self.op, np.ascontiguousarray(u, dtype=np.float64),
                                np.ascontiguousarray(rho_phys_active, dtype=np.float64), dc, float(penal))
        return dc

    def von_mises(self, u):
        out = np.zeros(self.fe.total_elements)
        lib().orc_von_mises(self.op, np.ascontiguousarray(u, dtype=np.float64), out)
        return out


def static_run(fe: FeModel, tolerance=1e-6, max_iterations=5000, warm_start=None, throw_on_non_convergence=True,
               reactions=True):
    m = Model(fe)
    n = fe.total_dofs
    u = np.zeros(n)
    rx = np.zeros(n) if reactions else None
    c = C.c_double(0)
    md = C.c_double(0)
    r = PcgRes()
    msg = C.create_string_buffer(512)
    ws = None if warm_start is None else np.ascontiguousarray(warm_start, dtype=np.float64)
    st = lib().orc_static_run(m.h, tolerance, max_iterations, None if ws is None else ws.ctypes.data,
                              0 if ws is None else ws.size, int(throw_on_non_convergence), u,
                              None if rx is None else rx.ctypes.data, C.byref(c), C.byref(md), C.byref(r), msg, 512)
    if st:
        _raise(st, msg)
    return StaticAnalysisResult(u, c.value, rx, md.value,
                                PcgResult(r.iterations, r.final_residual, bool(r.converged), 0.0,
                                          r.message.decode() or None))


class Filter:
    def __init__(self, grid, domain, active, rmin):
        self.n = int(len(active))
        self.h = lib().orc_filter_create(grid.nx, grid.ny, grid.nz, np.ascontiguousarray(domain, dtype=np.uint8),
                                         np.ascontiguousarray(active, dtype=np.int32), self.n, float(rmin))

    def __del__(self):
        try:
            lib().orc_filter_free(self.h)
        except Exception:
            pass

    def apply(self, x):
        out = np.zeros(self.n)
        lib().orc_filter_apply(self.h, np.ascontiguousarray(x, dtype=np.float64), out)
        return out

    def adjoint(self, x):
        out = np.zeros(self.n)
        lib().orc_filter_adjoint(self.h, np.ascontiguousarray(x, dtype=np.float64), out)
        return out

    @property
    def s(self):
        out = np.zeros(self.n)
        lib().orc_filter_s(self.h, out)
        return out

    @property
    def nnz(self):
        return int(lib().orc_filter_nnz(self.h))


def oc_update(rho, dc, s, passive, f, move=0.2, rho_min=1e-3, lambda_guess=1.0, max_bisect=60, vol_tol=1e-8):
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    out = np.zeros_like(rho)
    pas = None if passive is None else np.ascontiguousarray(passive, dtype=np.uint8)
    lam = lib().orc_oc_update(rho, np.ascontiguousarray(dc, dtype=np.float64), np.ascontiguousarray(s, dtype=np.float64),
                              None if pas is None else pas.ctypes.data, out, rho.size, f, move, rho_min, lambda_guess,
                              max_bisect, vol_tol)
    return out, lam


def oc_trace(rho, dc, s, passive, f, move=0.2, rho_min=1e-3, lambda_guess=1.0, max_bisect=60, vol_tol=1e-8):
    """The volume evaluations of OcOptimizer.Update in order: (lambdas, volumes, sum of s in element order)."""
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    pas = None if passive is None else np.ascontiguousarray(passive, dtype=np.uint8)
    cap = 512
    lam = np.zeros(cap)
    vol = np.zeros(cap)
    ts = C.c_double(0)
    k = lib().orc_oc_trace(rho, np.ascontiguousarray(dc, dtype=np.float64), np.ascontiguousarray(s, dtype=np.float64),
                           None if pas is None else pas.ctypes.data, rho.size, f, move, rho_min, lambda_guess,
                           max_bisect, vol_tol, lam, vol, cap, C.byref(ts))
    return lam[:k].copy(), vol[:k].copy(), ts.value


def heaviside_project(rho_tilde, beta, eta=0.5):
    """HeavisideProjection.Project (HeavisideProjection.cs:12-24)."""
    x = np.ascontiguousarray(rho_tilde, dtype=np.float64)
    out = np.empty_like(x)
    lib().orc_heaviside_project(x, out, x.size, beta, eta)
    return out


def heaviside_derivative(rho_tilde, beta, eta=0.5):
    """HeavisideProjection.Derivative (HeavisideProjection.cs:26-37)."""
    x = np.ascontiguousarray(rho_tilde, dtype=np.float64)
    out = np.empty_like(x)
    lib().orc_heaviside_derivative(x, out, x.size, beta, eta)
    return out


def quantized_frame(v):
    """RunWriter's 8-bit frame of a float density array and its FNV-1a checksum: (bytes, checksum)."""
    v = np.ascontiguousarray(v, dtype=np.float32)
    out = np.zeros(v.size, dtype=np.uint8)
    ck = lib().orc_quantized_checksum(v, v.size, out.ctypes.data)
    return out, int(ck)


def surface_nets(nx, ny, nz, density, h=1.0, origin=(0.0, 0.0, 0.0), threshold=0.5):
    """SurfaceNetsExtractor.Extract: (positions float32 [V,3], indices int32 [3T], info {passes, changes})."""
    L = lib()
    d = np.ascontiguousarray(density, dtype=np.float32)
    o = np.ascontiguousarray(origin, dtype=np.float32)
    L.orc_surface_nets.restype = C.c_void_p
    L.orc_surface_nets.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_void_p, C.c_void_p, C.c_float]
    L.orc_mesh_info.argtypes = [C.c_void_p, C.c_void_p]
    L.orc_mesh_copy.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_mesh_free.argtypes = [C.c_void_p]
    m = L.orc_surface_nets(nx, ny, nz, h, o.ctypes.data, d.ctypes.data, threshold)
    info = np.zeros(4, dtype=np.int64)
    L.orc_mesh_info(m, info.ctypes.data)
    pos = np.zeros((int(info[0]), 3), dtype=np.float32)
    idx = np.zeros(int(info[1]), dtype=np.int32)
    L.orc_mesh_copy(m, pos.ctypes.data, idx.ctypes.data)
    L.orc_mesh_free(m)
    return pos, idx, {"passes": int(info[2]), "changes": int(info[3])}


def taubin_smooth(positions, indices, iterations=3, lam=0.5, mu=-0.53):
    """TaubinSmoother.Smooth: smoothed copy of positions [V, 3] float32."""
    L = lib()
    p = np.array(positions, dtype=np.float32, copy=True, order="C")
    i = np.ascontiguousarray(indices, dtype=np.int32)
    L.orc_taubin_smooth.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int, C.c_float, C.c_float]
    L.orc_taubin_smooth(p.ctypes.data, p.shape[0], i.ctypes.data, i.size, iterations, lam, mu)
    return p


def passive_region(grid, nodes, radius=2):
    out = np.zeros(grid.total_elements, dtype=np.uint8)
    nodes = np.ascontiguousarray(nodes, dtype=np.int32)
    lib().orc_passive_region(grid.nx, grid.ny, grid.nz, nodes, nodes.size, radius, out)
    return out


@dataclass
class OracleSimpResult:
    records: list
    n_iters: int
    converged: bool
    u: np.ndarray
    phys: np.ndarray
    design: np.ndarray
    rho_phys_active: np.ndarray
    rho_design_active: np.ndarray
    lam: float


def topopt_run(fe: FeModel, o: OptimizerOptions) -> OracleSimpResult:
    m = Model(fe)
    keep = []

    def ptr(a, dt):
        if a is None:
            return None, 0
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data, a.size

    pm, pl = ptr(o.passive_mask, np.uint8)
    idp, idl = ptr(o.initial_density, np.float32)
    wp, wl = ptr(o.warm_start_displacements, np.float64)
    so = SimpOpts(o.volume_fraction, o.filter_radius_mm, o.penal, o.move_limit, o.max_iterations,
                  o.solver_tolerance_initial, o.solver_tolerance_final, o.solver_max_iterations, int(o.continuation),
                  int(o.enable_heaviside), o.rho_min, pm, pl, int(o.protect_boundary_hinges), idp, idl,
                  o.start_iteration, wp, wl, int(o.enforce_minimum_filter_radius), int(o.separate_load_cases))
    cap = max(1, o.max_iterations - o.start_iteration + 1)
    recs = (IterRec * cap)()
    ni = C.c_int32(0)
    cv = C.c_int32(0)
    n = fe.total_dofs
    na = fe.active_element_count
    u = np.zeros(n)
    phys = np.zeros(fe.total_elements, dtype=np.float32)
    des = np.zeros(fe.total_elements, dtype=np.float32)
    rpa = np.zeros(na)
    rda = np.zeros(na)
    lam = C.c_double(0)
    msg = C.create_string_buffer(512)
    st = lib().orc_topopt_run(m.h, C.byref(so), recs, cap, C.byref(ni), C.byref(cv), u, phys, des, rpa, rda,
                              C.byref(lam), msg, 512)
    if st:
        _raise(st, msg)
    rl = [dict(iteration=r.iteration, compliance=r.compliance, volume_fraction=r.volume_fraction,
               max_change=r.max_change, grey_level=r.grey_level, solver_iterations=r.solver_iterations,
               solver_residual=r.solver_residual, max_displacement=r.max_displacement) for r in recs[:ni.value]]
    return OracleSimpResult(rl, ni.value, bool(cv.value), u, phys, des, rpa, rda, lam.value)
