"""ctypes binding of libclgpu.so (declarations in include/clgpu.h).

The library is built in place by ``cuclarabel_b200.build``.  Loading fails
loudly when the shared object is missing: there is no CPU fallback.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libclgpu.so")

_lib = None

c_int = ctypes.c_int
c_double = ctypes.c_double
c_void_p = ctypes.c_void_p
c_ll = ctypes.c_longlong
dp = ctypes.POINTER(ctypes.c_double)
ip = ctypes.POINTER(ctypes.c_int)


class ClgpuSettings(ctypes.Structure):
    _fields_ = [
        ("max_iter", c_int), ("time_limit", c_double), ("max_step_fraction", c_double),
        ("tol_gap_abs", c_double), ("tol_gap_rel", c_double), ("tol_feas", c_double),
        ("tol_infeas_abs", c_double), ("tol_infeas_rel", c_double),
        ("tol_ktratio", c_double),
        ("reduced_tol_gap_abs", c_double), ("reduced_tol_gap_rel", c_double),
        ("reduced_tol_feas", c_double), ("reduced_tol_infeas_abs", c_double),
        ("reduced_tol_infeas_rel", c_double), ("reduced_tol_ktratio", c_double),
        ("equilibrate_enable", c_int), ("equilibrate_max_iter", c_int),
        ("equilibrate_min_scaling", c_double), ("equilibrate_max_scaling", c_double),
        ("linesearch_backtrack_step", c_double), ("min_switch_step_length", c_double),
        ("min_terminate_step_length", c_double),
        ("static_regularization_enable", c_int),
        ("static_regularization_constant", c_double),
        ("static_regularization_proportional", c_double),
        ("dynamic_regularization_enable", c_int),
        ("dynamic_regularization_eps", c_double),
        ("dynamic_regularization_delta", c_double),
        ("iterative_refinement_enable", c_int),
        ("iterative_refinement_reltol", c_double),
        ("iterative_refinement_abstol", c_double),
        ("iterative_refinement_max_iter", c_int),
        ("iterative_refinement_stop_ratio", c_double),
        ("direct_solve_method", c_int), ("soc_threshold", c_int), ("verbose", c_int),
        ("setup_threads", c_int), ("fused_solves", c_int), ("device_setup", c_int),
        ("autotune", c_int),
    ]


class ClgpuInfo(ctypes.Structure):
    _fields_ = [
        ("status", c_int), ("iterations", c_int),
        ("obj_val", c_double), ("obj_val_dual", c_double),
        ("cost_primal", c_double), ("cost_dual", c_double),
        ("res_primal", c_double), ("res_dual", c_double),
        ("res_primal_inf", c_double), ("res_dual_inf", c_double),
        ("gap_abs", c_double), ("gap_rel", c_double), ("ktratio", c_double),
        ("mu", c_double), ("sigma", c_double), ("step_length", c_double),
        ("solve_time", c_double),
    ]


class ClgpuProblem(ctypes.Structure):
    _fields_ = [
        ("n", c_int), ("m", c_int),
        ("Pp", ip), ("Pi", ip), ("Px", dp), ("q", dp),
        ("Ap", ip), ("Ai", ip), ("Ax", dp), ("b", dp),
        ("ncones", c_int), ("cone_types", ip), ("cone_dims", ip), ("cone_params", dp),
    ]


# every symbol declared in include/clgpu.h
EXPORTED = [
    "clgpu_default_settings", "clgpu_solver_create", "clgpu_solver_solve",
    "clgpu_solver_get_info", "clgpu_solver_get_solution", "clgpu_solver_get_solutions",
    "clgpu_solver_update_qb", "clgpu_solver_update_data", "clgpu_solver_device_bytes",
    "clgpu_solver_launch_count",
    "clgpu_solver_set_profiling", "clgpu_solver_get_profile", "clgpu_solver_get_phase_times",
    "clgpu_solver_get_phase_bytes",
    "clgpu_solver_destroy", "clgpu_serve_admit", "clgpu_serve_step", "clgpu_serve_collect",
    "clgpu_cones_create", "clgpu_cones_destroy", "clgpu_cones_numel", "clgpu_cones_degree",
    "clgpu_cones_hs_len", "clgpu_update_scaling", "clgpu_set_identity_scaling",
    "clgpu_get_Hs", "clgpu_mul_Hs", "clgpu_affine_ds", "clgpu_combined_ds_shift",
    "clgpu_ds_from_dz_offset", "clgpu_step_length", "clgpu_compute_barrier",
    "clgpu_margins", "clgpu_scaled_unit_shift", "clgpu_unit_initialization",
    "clgpu_debug_check_instance", "clgpu_debug_instance_path", "clgpu_debug_pinned_stats",
    "clgpu_debug_factor_stream",
    "clgpu_margins_static",
    "clgpu_cones_set_profiling", "clgpu_cones_last_kernel_ms",
    "clgpu_cones_get_launch_shapes", "clgpu_cones_set_launch_shapes",
    "clgpu_solver_get_launch_shapes", "clgpu_debug_soc_tiles",
    "clgpu_solver_get_solution_views",
    "clgpu_mul_Hs_diag", "clgpu_rectify_equilibration", "clgpu_refresh_kkt",
    "clgpu_step_length_device", "clgpu_ldl_create", "clgpu_ldl_refactor", "clgpu_ldl_solve",
    "clgpu_ldl_destroy", "clgpu_residuals", "clgpu_residuals_work_len", "clgpu_add_step",
    "clgpu_cones_debug_scaling", "clgpu_solver_get_sn_profile", "clgpu_solver_debug_setup",
    "clgpu_solver_get_sn_refinement",
]


def _declare(L):
    L.clgpu_default_settings.argtypes = [ctypes.POINTER(ClgpuSettings)]
    L.clgpu_solver_create.argtypes = [ctypes.POINTER(ClgpuProblem), c_int,
                                      ctypes.POINTER(ClgpuSettings), ctypes.POINTER(c_void_p)]
    L.clgpu_solver_solve.argtypes = [c_void_p, c_void_p]
    L.clgpu_solver_get_info.argtypes = [c_void_p, c_int, ctypes.POINTER(ClgpuInfo)]
    L.clgpu_solver_get_solution.argtypes = [c_void_p, c_int, dp, dp, dp]
    L.clgpu_solver_get_solutions.argtypes = [c_void_p, dp, dp, dp, ctypes.POINTER(ClgpuInfo)]
    L.clgpu_solver_update_qb.argtypes = [c_void_p, c_int, dp, dp]
    L.clgpu_solver_update_data.argtypes = [c_void_p, dp, dp, dp, dp, c_void_p]
    L.clgpu_solver_device_bytes.argtypes = [c_void_p]
    L.clgpu_solver_device_bytes.restype = c_ll
    L.clgpu_solver_launch_count.argtypes = [c_void_p]
    L.clgpu_solver_launch_count.restype = c_ll
    L.clgpu_solver_set_profiling.argtypes = [c_void_p, c_int]
    L.clgpu_solver_get_profile.argtypes = [c_void_p, dp, dp, dp, dp, dp, ip]
    L.clgpu_solver_get_phase_times.argtypes = [c_void_p, dp, ctypes.POINTER(c_ll)]
    L.clgpu_solver_get_phase_bytes.argtypes = [c_void_p, dp]
    L.clgpu_solver_destroy.argtypes = [c_void_p]
    L.clgpu_serve_admit.argtypes = [c_void_p, ip, c_int, dp, dp, c_void_p]
    L.clgpu_serve_step.argtypes = [c_void_p, c_void_p, ip, ip, ip]
    L.clgpu_serve_collect.argtypes = [c_void_p, ip, c_int, dp, dp, dp,
                                      ctypes.POINTER(ClgpuInfo), c_void_p]
    L.clgpu_cones_create.argtypes = [c_int, ip, ip, dp, c_int, ctypes.POINTER(c_void_p)]
    L.clgpu_cones_destroy.argtypes = [c_void_p]
    for f in ("clgpu_cones_numel", "clgpu_cones_degree", "clgpu_cones_hs_len"):
        getattr(L, f).argtypes = [c_void_p]
    L.clgpu_cones_set_profiling.argtypes = [c_void_p, c_int]
    L.clgpu_cones_get_launch_shapes.argtypes = [c_void_p, ip, ip]
    L.clgpu_cones_set_launch_shapes.argtypes = [c_void_p, c_int, ip]
    L.clgpu_solver_get_launch_shapes.argtypes = [c_void_p, ip, ip]
    L.clgpu_debug_soc_tiles.argtypes = [ip, ip, c_int, c_int, c_int, ip, c_int]
    L.clgpu_solver_get_solution_views.argtypes = [c_void_p, ctypes.POINTER(dp),
                                                  ctypes.POINTER(dp), ctypes.POINTER(dp)]
    L.clgpu_cones_last_kernel_ms.argtypes = [c_void_p, dp]
    V = c_void_p  # device pointers are passed as integers
    L.clgpu_update_scaling.argtypes = [c_void_p, V, V, c_double, c_int, c_void_p]
    L.clgpu_set_identity_scaling.argtypes = [c_void_p, c_void_p]
    L.clgpu_get_Hs.argtypes = [c_void_p, V, c_void_p]
    L.clgpu_mul_Hs.argtypes = [c_void_p, V, V, c_void_p]
    L.clgpu_affine_ds.argtypes = [c_void_p, V, V, c_void_p]
    L.clgpu_combined_ds_shift.argtypes = [c_void_p, V, V, V, V, c_double, c_void_p]
    L.clgpu_ds_from_dz_offset.argtypes = [c_void_p, V, V, V, c_void_p]
    L.clgpu_step_length.argtypes = [c_void_p, V, V, V, V, c_double, c_double, c_double,
                                    c_double, dp, c_void_p]
    L.clgpu_compute_barrier.argtypes = [c_void_p, V, V, V, V, c_double, dp, c_void_p]
    L.clgpu_margins.argtypes = [c_void_p, V, c_int, dp, dp, c_void_p]
    L.clgpu_margins_static.argtypes = [c_int, ip, ip, V, c_int, dp, dp, c_void_p]
    L.clgpu_scaled_unit_shift.argtypes = [c_void_p, V, c_double, c_int, c_void_p]
    L.clgpu_unit_initialization.argtypes = [c_void_p, V, V, c_void_p]
    L.clgpu_debug_check_instance.argtypes = [ctypes.POINTER(ClgpuProblem),
                                             ctypes.POINTER(ClgpuSettings), dp]
    L.clgpu_debug_instance_path.argtypes = [ctypes.POINTER(ClgpuProblem),
                                            ctypes.POINTER(ClgpuSettings), ip,
                                            ctypes.POINTER(ctypes.c_longlong)]
    L.clgpu_debug_pinned_stats.argtypes = [ctypes.POINTER(ctypes.c_longlong)]
    L.clgpu_debug_factor_stream.argtypes = [ctypes.POINTER(ClgpuProblem),
                                            ctypes.POINTER(ClgpuSettings), dp]
    # KKT-level boundary (device pointers as integers)
    L.clgpu_mul_Hs_diag.argtypes = [c_void_p, V, V, c_void_p]
    L.clgpu_rectify_equilibration.argtypes = [c_void_p, V, V, ip, c_void_p]
    L.clgpu_refresh_kkt.argtypes = [c_void_p, V, V, V, V, V, V, c_void_p]
    L.clgpu_step_length_device.argtypes = [c_void_p, V, V, V, V, V, c_double, c_double,
                                           c_double, V, c_void_p]
    L.clgpu_ldl_create.argtypes = [c_int, ip, ip, ctypes.POINTER(ctypes.c_byte),
                                   ctypes.POINTER(ClgpuSettings), ctypes.POINTER(c_void_p)]
    L.clgpu_ldl_refactor.argtypes = [c_void_p, V, dp, c_void_p]
    L.clgpu_ldl_solve.argtypes = [c_void_p, V, V, c_void_p]
    L.clgpu_ldl_destroy.argtypes = [c_void_p]
    L.clgpu_residuals.argtypes = [c_int, c_int] + [V] * 9 + [V] * 7 + [V] * 7 + [c_void_p]
    L.clgpu_residuals_work_len.argtypes = []
    L.clgpu_add_step.argtypes = [c_int, c_int] + [V] * 11 + [c_void_p]
    L.clgpu_cones_debug_scaling.argtypes = [c_void_p] + [dp] * 9 + [ip]
    L.clgpu_solver_get_sn_profile.argtypes = [c_void_p, dp, dp, ctypes.POINTER(c_ll)]
    L.clgpu_solver_get_sn_refinement.argtypes = [c_void_p, ctypes.POINTER(c_ll), dp]
    L.clgpu_solver_debug_setup.argtypes = [c_void_p, dp, dp, dp, dp, dp, dp,
                                           ctypes.POINTER(c_ll)]


def load():
    """Load libclgpu.so; raises if it is missing (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "libclgpu.so is not built (%s); run `python -m cuclarabel_b200.build`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib
