"""ctypes binding of libmycel_b200.so (the C ABI declared in include/mycel.h).

The shared library is built in-tree (python -m mycel_b200.build). There is no fallback: if the library is
missing or has no CUDA device, calls fail with an error instead of computing anything elsewhere.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmycel_b200.so")

P = C.c_void_p
i32 = C.c_int32
i64 = C.c_int64
dbl = C.c_double


class Grid(C.Structure):
    _fields_ = [("nx", i32), ("ny", i32), ("nz", i32), ("h", C.c_float)]


class Material(C.Structure):
    _fields_ = [("e0", dbl), ("nu", dbl), ("emin_ratio", dbl)]


class LoadCaseC(C.Structure):
    _fields_ = [("n_nodes", i32), ("nodes", P), ("node_area", P), ("force", C.c_float * 3)]


class ProblemInfo(C.Structure):
    _fields_ = [("total_elements", i64), ("total_nodes", i64), ("total_dofs", i64), ("active_elements", i64),
                ("active_nodes", i64), ("active_fixed_dofs", i64), ("device_bytes", i64)]


class PcgResultC(C.Structure):
    _fields_ = [("iterations", i32), ("final_residual", dbl), ("converged", i32), ("elapsed_ms", dbl),
                ("refinement_steps", i32), ("inner_iterations", i32), ("message", C.c_char * 256),
                ("fallback_iterations", i32)]


class StaticOptions(C.Structure):
    _fields_ = [("tolerance", dbl), ("max_iterations", i32), ("throw_on_non_convergence", i32), ("precision", i32)]


class SimpOptions(C.Structure):
    _fields_ = [("volume_fraction", dbl), ("filter_radius_mm", dbl), ("penal", dbl), ("move_limit", dbl),
                ("max_iterations", i32), ("solver_tolerance_initial", dbl), ("solver_tolerance_final", dbl),
                ("solver_max_iterations", i32), ("continuation", i32), ("enable_heaviside", i32), ("rho_min", dbl),
                ("passive_mask", P), ("passive_mask_len", i64), ("protect_boundary_hinges", i32),
                ("initial_density", P), ("initial_density_len", i64), ("start_iteration", i32),
                ("warm_start_displacements", P), ("warm_start_len", i64), ("enforce_minimum_filter_radius", i32),
                ("precision", i32), ("separate_load_cases", i32)]


class IterRecord(C.Structure):
    _fields_ = [("iteration", i32), ("compliance", dbl), ("volume_fraction", dbl), ("max_change", dbl),
                ("grey_level", dbl), ("solver_iterations", i32), ("solver_residual", dbl), ("max_displacement", dbl),
                ("solve_ms", dbl), ("sensitivity_ms", dbl), ("filter_ms", dbl), ("update_ms", dbl), ("total_ms", dbl),
                ("refinement_steps", i32)]


PROGRESS_FN = C.CFUNCTYPE(None, P, C.POINTER(IterRecord), C.POINTER(C.c_float), C.POINTER(C.c_float))


class ServerOptions(C.Structure):
    _fields_ = [("device", i32), ("slots", i32), ("hbm_budget_bytes", i64)]


class JobSpec(C.Structure):
    _fields_ = [("grid", Grid), ("domain", P), ("material", Material), ("fixed_dofs", P), ("n_fixed", i32),
                ("loads", P), ("n_loads", i32), ("element_density", P), ("penal", dbl), ("options", SimpOptions),
                ("keep_u", i32)]


class JobInfo(C.Structure):
    _fields_ = [("state", i32), ("status", i32), ("iterations", i32), ("converged", i32), ("device_bytes", i64),
                ("submit_s", dbl), ("start_s", dbl), ("finish_s", dbl), ("final_compliance", dbl),
                ("solver_iterations", i64), ("message", C.c_char * 256)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", i64), ("completed", i64), ("failed", i64), ("running", i64), ("queued", i64),
                ("simp_iterations", i64), ("first_submit_s", dbl), ("last_finish_s", dbl), ("p50_latency_s", dbl),
                ("p99_latency_s", dbl), ("mean_latency_s", dbl), ("max_latency_s", dbl), ("p50_queue_s", dbl),
                ("p99_queue_s", dbl), ("admitted_bytes", i64), ("peak_admitted_bytes", i64)]

# name -> (restype, argtypes); exactly the entry points of include/mycel.h
SIGNATURES = {
    "mycel_version": (i32, []),
    "mycel_ctx_create": (i32, [i32, C.POINTER(P)]),
    "mycel_ctx_destroy": (i32, [P]),
    "mycel_ctx_stream": (P, [P]),
    "mycel_last_error": (C.c_char_p, [P]),
    "mycel_ctx_launch_count": (i64, [P]),
    "mycel_ctx_packed_count": (i64, [P]),
    "mycel_ctx_set_profiling": (i32, [P, i32]),
    "mycel_ctx_set_oc_wait": (i32, [P, i64, i32]),
    "mycel_problem_kernel_bench": (i32, [P, i32, i32, C.POINTER(dbl)]),
    "mycel_ctx_kernel_timing": (i32, [P, i32, C.POINTER(dbl), C.POINTER(i64), C.POINTER(i64), C.POINTER(i64)]),
    "mycel_problem_create": (i32, [P, C.POINTER(Grid), P, C.POINTER(Material), P, i32, P, i32, P, dbl,
                                   C.POINTER(P)]),
    "mycel_problem_destroy": (i32, [P]),
    "mycel_problem_info_get": (i32, [P, C.POINTER(ProblemInfo)]),
    "mycel_problem_forces": (i32, [P, P]),
    "mycel_problem_load_cases": (i32, [P, C.POINTER(i32)]),
    "mycel_problem_case_forces": (i32, [P, i32, P]),
    "mycel_problem_set_tuning": (i32, [P, i32, i32]),
    "mycel_problem_get_tuning": (i32, [P, i32, C.POINTER(i32)]),
    "mycel_update_densities": (i32, [P, P, dbl]),
    "mycel_diagonal": (i32, [P, P]),
    "mycel_apply_k": (i32, [P, P, P, i32, i32]),
    "mycel_pcg_solve": (i32, [P, P, P, dbl, i32, i32, C.POINTER(PcgResultC)]),
    "mycel_static_solve": (i32, [P, C.POINTER(StaticOptions), P, i64, P, P, P, C.POINTER(dbl), C.POINTER(dbl),
                                 C.POINTER(PcgResultC)]),
    "mycel_static_solve_cases": (i32, [P, C.POINTER(StaticOptions), P, P, P, P]),
    "mycel_filter_create": (i32, [P, dbl, C.POINTER(P)]),
    "mycel_filter_destroy": (i32, [P]),
    "mycel_filter_apply": (i32, [P, P, P]),
    "mycel_filter_adjoint": (i32, [P, P, P]),
    "mycel_filter_s": (i32, [P, P]),
    "mycel_sensitivities": (i32, [P, P, P, dbl, P]),
    "mycel_oc_update": (i32, [P, i32, P, P, P, P, P, dbl, dbl, dbl, dbl, i32, dbl, C.POINTER(dbl)]),
    "mycel_pow": (i32, [P, i64, P, P, i64, P]),
    "mycel_oc_update_noalloc": (i32, [P, i32, P, P, P, P, P, dbl, dbl, dbl, dbl, i32, dbl, C.POINTER(dbl)]),
    "mycel_heaviside_project": (i32, [P, i64, P, P, dbl, dbl]),
    "mycel_heaviside_derivative": (i32, [P, i64, P, P, dbl, dbl]),
    "mycel_simp_run": (i32, [P, C.POINTER(SimpOptions), PROGRESS_FN, P, P, P, C.POINTER(IterRecord), i32,
                             C.POINTER(i32), C.POINTER(i32), P, P, P]),
    "mycel_simp_begin": (i32, [P, C.POINTER(SimpOptions), C.POINTER(P)]),
    "mycel_simp_step": (i32, [P, C.POINTER(IterRecord), C.POINTER(i32)]),
    "mycel_simp_step_many": (i32, [C.POINTER(P), i32, C.POINTER(IterRecord), C.POINTER(i32), C.POINTER(i32), P]),
    "mycel_simp_converged": (i32, [P]),
    "mycel_simp_run_many": (i32, [C.POINTER(P), i32, C.POINTER(IterRecord), i32, C.POINTER(i32), C.POINTER(i32), P]),
    "mycel_simp_read": (i32, [P, P, P, P, P, P, C.POINTER(dbl)]),
    "mycel_simp_end": (i32, [P]),
    "mycel_simp_frame_begin": (i32, [P, C.POINTER(i32)]),
    "mycel_simp_frame_end": (i32, [P, i32, P, P, C.POINTER(C.c_uint32)]),
    "mycel_server_create": (i32, [C.POINTER(ServerOptions), C.POINTER(P)]),
    "mycel_server_submit": (i32, [P, C.POINTER(JobSpec), C.POINTER(i64)]),
    "mycel_server_job_info": (i32, [P, i64, C.POINTER(JobInfo)]),
    "mycel_server_wait": (i32, [P, i64, dbl]),
    "mycel_server_job_result": (i32, [P, i64, C.POINTER(IterRecord), i32, P, P, P]),
    "mycel_server_stats_get": (i32, [P, C.POINTER(ServerStats)]),
    "mycel_server_destroy": (i32, [P]),
    "mycel_server_last_error": (C.c_char_p, [P]),
    "mycel_job_device_bytes": (i64, [C.POINTER(JobSpec)]),
    "mycel_average_element_to_node": (i32, [P, P, i64, P]),
    "mycel_surface_nets": (i32, [P, i32, i32, i32, C.c_float, P, P, i64, C.c_float, C.POINTER(P)]),
    "mycel_simp_surface_nets": (i32, [P, P, C.c_float, C.POINTER(P)]),
    "mycel_mesh_info": (i32, [P, C.POINTER(i64), C.POINTER(i64), C.POINTER(i32), C.POINTER(i64)]),
    "mycel_mesh_copy": (i32, [P, P, P]),
    "mycel_mesh_destroy": (None, [P]),
    "mycel_taubin_smooth": (i32, [P, P, i64, P, i64, i32, C.c_float, C.c_float]),
}

_lib = None


def load() -> C.CDLL:
    """Load the in-tree library; raises ImportError if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libmycel_b200.so not found at {LIB_PATH}; build it with `python -m mycel_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(a):
    return None if a is None else a.ctypes.data


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)
