"""ctypes binding of the C ABI in include/hicarw.h (libhicarw.so, built in-tree).

The library is the product: there is no CPU fallback.  Loading fails loudly
when the shared library is missing or cannot be loaded.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libhicarw.so")

HICARW_OK, HICARW_ITER_CAP, HICARW_BREAKDOWN, HICARW_FELL_BACK = 0, 1, 2, 3
ERRORS = {-1: "HICARW_ERR_ARG", -2: "HICARW_ERR_STATE", -3: "HICARW_ERR_CUDA", -4: "HICARW_ERR_DIVERGED",
          -5: "HICARW_ERR_NAN", -6: "HICARW_ERR_TIMEOUT"}
MEM_DEVICE, MEM_HOST = 0, 1
KRYLOV_F64, KRYLOV_F32, KRYLOV_F32_X64 = 0, 1, 2
SOLVER_REFERENCE, SOLVER_FUSED, SOLVER_MIXED, SOLVER_FGMRES = 0, 1, 2, 3
CRIT_RECURRENCE, CRIT_TRUE = 0, 1
PRECOND_JACOBI, PRECOND_MG, PRECOND_LEARNED, PRECOND_MG_LEARNED = 0, 1, 2, 3

# Every exported symbol of include/hicarw.h (checked by the CPU test suite).
EXPORTS = [
    "hicarw_default_options", "hicarw_init_iter_winds", "hicarw_finalize_iter_winds", "hicarw_calc_iter_winds",
    "hicarw_calc_divergence", "hicarw_probe_lambda_pattern", "hicarw_probe_zero_corrections",
    "hicarw_probe_apply_corrections", "hicarw_probe_record", "hicarw_probe_finalize",
    "hicarw_calibrate_projection_operator", "hicarw_reset_solution", "hicarw_get_lambda", "hicarw_get_coefs",
    "hicarw_set_coefs", "hicarw_apply_operator", "hicarw_apply_precond", "hicarw_solve_rhs", "hicarw_set_options",
    "hicarw_get_history", "hicarw_last_error", "hicarw_kernel_launches", "hicarw_mg_tma_launches", "hicarw_profile_iteration",
    "hicarw_residual_norm_noalloc", "hicarw_nn_act_pitch", "hicarw_nn_conv3", "hicarw_nn_conv3_wgrad",
    "hicarw_nn_conv3_time",
    "hicarw_unet_create", "hicarw_unet_destroy", "hicarw_unet_grid", "hicarw_unet_num_params",
    "hicarw_unet_get_params", "hicarw_unet_set_params", "hicarw_unet_get_grads", "hicarw_unet_zero_grads",
    "hicarw_unet_features", "hicarw_unet_forward", "hicarw_unet_backward", "hicarw_unet_backward_residual",
    "hicarw_unet_adam_step", "hicarw_unet_apply", "hicarw_set_learned_precond",
    "hicarw_batch_create", "hicarw_batch_destroy", "hicarw_batch_config", "hicarw_batch_get_config",
    "hicarw_batch_calc_iter_winds", "hicarw_batch_autotune", "hicarw_batch_latencies",
    "hicarw_calc_w_real", "hicarw_calc_idealized_wgrid", "hicarw_balance_uvw", "hicarw_calc_alpha",
    "hicarw_smooth_alpha", "hicarw_update_stability", "hicarw_debug_wait_timeout",
    "hicarw_set_kernel_tuning", "hicarw_dist_configure", "hicarw_dist_setup", "hicarw_dist_apply",
    "hicarw_dist_precond", "hicarw_dist_face", "hicarw_dist_spmv", "hicarw_dist_update", "hicarw_dist_state",
]


class BatchItem(C.Structure):
    _fields_ = [("alpha", C.c_void_p), ("div", C.c_void_p), ("density", C.c_void_p),
                ("u", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p)]


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("dx", C.c_float), ("nest", C.c_int)]


class Options(C.Structure):
    _fields_ = [("max_iters", C.c_int), ("verbose", C.c_int), ("tol_rel", C.c_double), ("tol_abs", C.c_double),
                ("krylov_precision", C.c_int), ("solver", C.c_int), ("criterion", C.c_int),
                ("replace_every", C.c_int), ("check_every", C.c_int), ("precond", C.c_int),
                ("stall_iters", C.c_int), ("mg_omega", C.c_float), ("fgmres_restart", C.c_int),
                ("mg_coarse_scale", C.c_float), ("mg_skip_fine_presmooth", C.c_int),
                ("mg_w_levels", C.c_int), ("mg_precision", C.c_int)]


METRIC_FIELDS = ["jacobian", "jacobian_u", "jacobian_v", "jacobian_w", "dzdx", "dzdy", "dzdx_u", "dzdy_v",
                 "advection_dz", "neighbor_terrain", "mapfac_mx_u", "mapfac_my_v", "mapfac_my_u", "mapfac_mx_v",
                 "mapfac_mxy"]


class Metrics(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in METRIC_FIELDS]


class Stats(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("sweeps", C.c_int), ("retries", C.c_int),
                ("res0", C.c_double), ("res_final", C.c_double), ("b_norm", C.c_double), ("target", C.c_double),
                ("true_res", C.c_double), ("replacements", C.c_int), ("launches", C.c_int),
                ("precond", C.c_int), ("solve_ms", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class HicarwError(RuntimeError):
    pass


_LIB = None


def load(path: str = LIB_PATH):
    """Load libhicarw.so (raise if it is absent: the CUDA library is the only implementation)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise HicarwError(f"{path} is missing: build it with `python -m hicar_b200.build` "
                          f"(the wind solver has no CPU fallback)")
    lib = C.CDLL(path)
    vp, ci, cf = C.c_void_p, C.c_int, C.c_float
    P = C.POINTER
    sig = {
        "hicarw_default_options": (None, [P(Options)]),
        "hicarw_init_iter_winds": (ci, [P(Grid), P(Options), P(Metrics), ci, vp, P(vp)]),
        "hicarw_finalize_iter_winds": (ci, [vp]),
        "hicarw_calc_iter_winds": (ci, [vp, vp, vp, vp, ci, vp, vp, vp, ci, vp, P(Stats)]),
        "hicarw_calc_divergence": (ci, [vp, vp, vp, vp, vp, vp, ci, ci, ci, ci, vp]),
        "hicarw_probe_lambda_pattern": (ci, [vp, ci, ci, ci, vp]),
        "hicarw_probe_zero_corrections": (ci, [vp, vp, vp, vp, ci, vp]),
        "hicarw_probe_apply_corrections": (ci, [vp, vp, vp, ci, vp, vp, vp, ci, vp]),
        "hicarw_probe_record": (ci, [vp, vp, ci, ci, ci, P(cf), ci, vp]),
        "hicarw_probe_finalize": (ci, [vp, cf, vp]),
        "hicarw_calibrate_projection_operator": (ci, [vp, vp, vp, ci, vp, vp, vp, P(cf), ci, vp]),
        "hicarw_reset_solution": (ci, [vp, vp]),
        "hicarw_get_lambda": (ci, [vp, vp, ci, vp]),
        "hicarw_get_coefs": (ci, [vp, vp, ci, vp]),
        "hicarw_set_coefs": (ci, [vp, vp, ci, ci, vp]),
        "hicarw_apply_operator": (ci, [vp, vp, vp, ci, vp]),
        "hicarw_apply_precond": (ci, [vp, vp, vp, ci, ci, vp]),
        "hicarw_solve_rhs": (ci, [vp, vp, ci, vp, P(Stats)]),
        "hicarw_set_options": (ci, [vp, P(Options)]),
        "hicarw_get_history": (ci, [vp, vp, ci]),
        "hicarw_last_error": (C.c_char_p, [vp]),
        "hicarw_kernel_launches": (C.c_longlong, []),
        "hicarw_mg_tma_launches": (C.c_longlong, []),
        "hicarw_profile_iteration": (ci, [vp, ci, vp, vp, vp, vp, ci, vp]),
        "hicarw_residual_norm_noalloc": (ci, [vp, vp, vp, vp, vp]),
        "hicarw_nn_act_pitch": (ci, [ci]),
        "hicarw_nn_conv3": (ci, [ci, ci, ci, ci, ci, vp, vp, vp, vp, vp, ci, ci, vp, vp, vp]),
        "hicarw_nn_conv3_wgrad": (ci, [ci, ci, ci, ci, ci, vp, vp, vp, vp, vp]),
        "hicarw_nn_conv3_time": (ci, [ci, ci, ci, ci, ci, vp, vp, vp, vp, ci, vp, P(C.c_float)]),
        "hicarw_unet_create": (ci, [ci, ci, ci, C.c_ulonglong, P(vp)]),
        "hicarw_unet_destroy": (ci, [vp]),
        "hicarw_unet_grid": (ci, [vp, P(ci), P(ci), P(ci)]),
        "hicarw_unet_num_params": (C.c_longlong, [vp]),
        "hicarw_unet_get_params": (ci, [vp, vp, ci, vp]),
        "hicarw_unet_set_params": (ci, [vp, vp, ci, vp]),
        "hicarw_unet_get_grads": (ci, [vp, vp, ci, vp]),
        "hicarw_unet_zero_grads": (ci, [vp, vp]),
        "hicarw_unet_features": (ci, [vp, vp, vp, vp, P(C.c_float), vp]),
        "hicarw_unet_forward": (ci, [vp, vp, vp, vp]),
        "hicarw_unet_backward": (ci, [vp, vp, C.c_float, P(C.c_float), vp]),
        "hicarw_unet_backward_residual": (ci, [vp, vp, vp, C.c_float, P(C.c_float), vp]),
        "hicarw_unet_adam_step": (ci, [vp, C.c_float, vp]),
        "hicarw_unet_apply": (ci, [vp, vp, vp, vp, vp]),
        "hicarw_set_learned_precond": (ci, [vp, vp]),
        "hicarw_batch_create": (ci, [ci, vp, P(vp)]),
        "hicarw_batch_destroy": (ci, [vp]),
        "hicarw_batch_config": (ci, [vp, ci, ci]),
        "hicarw_batch_get_config": (ci, [vp, P(ci), P(ci)]),
        "hicarw_batch_calc_iter_winds": (ci, [vp, P(BatchItem), ci, ci, vp, P(Stats)]),
        "hicarw_batch_autotune": (ci, [vp, P(BatchItem), ci, vp, P(C.c_double)]),
        "hicarw_batch_latencies": (ci, [vp, vp]),
        "hicarw_calc_w_real": (ci, [vp, vp, vp, vp, vp, ci, vp]),
        "hicarw_calc_idealized_wgrid": (ci, [vp, vp, vp, vp, vp, ci, vp]),
        "hicarw_balance_uvw": (ci, [vp, vp, vp, vp, vp, ci, ci, ci, vp]),
        "hicarw_calc_alpha": (ci, [vp, vp, vp, ci, ci, vp]),
        "hicarw_smooth_alpha": (ci, [vp, vp, ci, ci, ci, vp]),
        "hicarw_update_stability": (ci, [vp, vp, vp, vp, vp, vp, ci, ci, vp, vp, ci, vp]),
        "hicarw_debug_wait_timeout": (ci, [vp, C.c_double, vp]),
        "hicarw_set_kernel_tuning": (ci, [vp, ci, ci]),
        "hicarw_dist_configure": (ci, [vp, ci]),
        "hicarw_dist_setup": (ci, [vp, vp, vp, ci, vp]),
        "hicarw_dist_apply": (ci, [vp, ci, vp, ci, vp]),
        "hicarw_dist_precond": (ci, [vp, ci, vp]),
        "hicarw_dist_face": (ci, [vp, ci, ci, vp, ci, vp]),
        "hicarw_dist_spmv": (ci, [vp, ci, vp, ci, vp]),
        "hicarw_dist_update": (ci, [vp, vp]),
        "hicarw_dist_state": (ci, [vp, P(ci), P(Stats), vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def default_options() -> Options:
    o = Options()
    load().hicarw_default_options(C.byref(o))
    return o


def check(rc: int, handle=None, allow_status: bool = True) -> int:
    if rc < 0:
        msg = load().hicarw_last_error(handle).decode()  # NULL handle: the calls without one (batches)
        raise HicarwError(f"{ERRORS.get(rc, rc)}: {msg}")
    return rc
