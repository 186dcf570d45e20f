"""ctypes binding of liblaminocam_b200.so (the C ABI in include/laminocam.h)."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblaminocam_b200.so")


class SolverParams(C.Structure):
    _fields_ = [("max_iters", C.c_int), ("inner_iters", C.c_int), ("tol", C.c_float),
                ("xtol", C.c_float), ("lambda_", C.c_float), ("mu", C.c_float),
                ("fp32_scalars", C.c_int), ("poll_every", C.c_int), ("use_graph", C.c_int),
                ("residual_refresh", C.c_int)]


class SolverStats(C.Structure):
    _fields_ = [("iters", C.c_int), ("cg_iters_total", C.c_int), ("residual", C.c_double),
                ("dx", C.c_double), ("stop_reason", C.c_int), ("elapsed_ms", C.c_double)]


class ReconParamsC(C.Structure):
    _fields_ = [("method", C.c_int), ("solver", SolverParams), ("nufft_tol", C.c_double),
                ("pad_factor", C.c_float), ("psf_fp32", C.c_int)]


class ProfileEntry(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("count", C.c_long), ("total_ms", C.c_double),
                ("bytes", C.c_double)]


class ServerParams(C.Structure):
    _fields_ = [("device", C.c_int), ("workers", C.c_int), ("hbm_budget_bytes", C.c_double),
                ("psf_cache_bytes", C.c_double), ("psf_cache", C.c_int), ("backfill", C.c_int),
                ("priority_2d", C.c_int)]


class JobInfo(C.Structure):
    _fields_ = [("queue_ms", C.c_double), ("run_ms", C.c_double), ("latency_ms", C.c_double),
                ("psf_hit", C.c_int), ("worker", C.c_int), ("device_bytes", C.c_double),
                ("error", C.c_char * 160)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_long), ("failed", C.c_long), ("queued", C.c_long),
                ("running", C.c_long), ("peak_running", C.c_long), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("span_s", C.c_double),
                ("recons_per_s", C.c_double), ("hbm_budget_bytes", C.c_double),
                ("peak_admitted_bytes", C.c_double), ("psf_hits", C.c_long),
                ("psf_misses", C.c_long), ("psf_cache_entries", C.c_long),
                ("psf_cache_bytes", C.c_double), ("p50_2d_ms", C.c_double), ("p99_2d_ms", C.c_double),
                ("p50_3d_ms", C.c_double), ("p99_3d_ms", C.c_double), ("backfilled", C.c_long)]


class Job2D(C.Structure):
    _fields_ = [("sinogram", C.POINTER(C.c_float)), ("ntheta", C.c_int), ("nradial", C.c_int),
                ("theta", C.POINTER(C.c_double)), ("n", C.c_int), ("recon", C.POINTER(C.c_float))]


OperatorFn = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_void_p)

vp = C.c_void_p
i32 = C.c_int
f64 = C.c_double
dptr = C.POINTER(C.c_double)
fptr = C.POINTER(C.c_float)

# name -> (restype, argtypes); must match include/laminocam.h
SIGNATURES = {
    "lc_version": (i32, []),
    "lc_context_create": (i32, [i32, vp, C.POINTER(vp)]),
    "lc_context_destroy": (i32, [vp]),
    "lc_context_set_stream": (i32, [vp, vp]),
    "lc_context_synchronize": (i32, [vp]),
    "lc_last_error": (C.c_char_p, [vp]),
    "lc_geometry2d_create": (i32, [vp, dptr, i32, i32, C.POINTER(vp)]),
    "lc_geometry3d_create": (i32, [vp, dptr, dptr, dptr, fptr, i32, i32, i32, C.POINTER(vp)]),
    "lc_geometry_destroy": (i32, [vp]),
    "lc_forward2d": (i32, [vp, vp, vp, i32, i32, i32, vp, f64]),
    "lc_backproj2d": (i32, [vp, vp, vp, i32, i32, i32, vp, f64]),
    "lc_sysmat2d_nufft": (i32, [vp, vp, vp, i32, i32, i32, vp, f64]),
    "lc_forward3d": (i32, [vp, vp, vp, i32, i32, i32, vp, f64]),
    "lc_backproj3d": (i32, [vp, vp, vp, i32, i32, i32, i32, vp, f64]),
    "lc_sysmat3d_nufft": (i32, [vp, vp, vp, i32, i32, i32, vp, f64]),
    "lc_psf_create": (i32, [vp, vp, i32, i32, i32, C.POINTER(vp)]),
    "lc_psf_create_ex": (i32, [vp, vp, i32, i32, i32, i32, C.POINTER(vp)]),
    "lc_psf_destroy": (i32, [vp]),
    "lc_psf_info": (i32, [vp, C.POINTER(C.c_int), C.POINTER(C.c_long)]),
    "lc_psf_kernel": (i32, [vp, vp, dptr]),
    "lc_psf_spectrum": (i32, [vp, vp, fptr]),
    "lc_sysmat_toeplitz": (i32, [vp, vp, vp, vp]),
    "lc_solver_params_default": (None, [C.POINTER(SolverParams)]),
    "lc_recon_params_default": (None, [C.POINTER(ReconParamsC)]),
    "lc_cgsolver": (i32, [vp, vp, vp, vp, C.POINTER(SolverParams), C.POINTER(SolverStats)]),
    "lc_split_bregman": (i32, [vp, vp, vp, vp, C.POINTER(SolverParams), C.POINTER(SolverStats)]),
    "lc_mbir2d": (i32, [vp, fptr, i32, i32, i32, dptr, C.POINTER(C.c_int), C.POINTER(ReconParamsC),
                        fptr, C.POINTER(SolverStats)]),
    "lc_mbir3d": (i32, [vp, fptr, i32, i32, i32, dptr, dptr, dptr, fptr, C.POINTER(C.c_int),
                        C.POINTER(ReconParamsC), fptr, C.POINTER(SolverStats)]),
    "lc_mbir3d_device": (i32, [vp, vp, i32, i32, i32, dptr, dptr, dptr, fptr, C.POINTER(C.c_int),
                               C.POINTER(ReconParamsC), vp, C.POINTER(SolverStats)]),
    "lc_cgsolver_op": (i32, [vp, OperatorFn, vp, C.c_long, vp, vp, C.POINTER(SolverParams),
                             C.POINTER(SolverStats)]),
    "lc_split_bregman_op": (i32, [vp, OperatorFn, vp, C.POINTER(C.c_int), vp, vp, C.POINTER(SolverParams),
                                  C.POINTER(SolverStats)]),
    "lc_mbir2d_batch": (i32, [vp, C.POINTER(Job2D), i32, C.POINTER(ReconParamsC), i32,
                              C.POINTER(SolverStats)]),
    "lc_profile_enable": (i32, [vp, i32]),
    "lc_kernel_launches": (C.c_long, []),
    "lc_sysmat2d_toeplitz_noalloc": (i32, [vp, vp, i32, vp, vp, i32, i32]),
    "lc_profile_read": (i32, [vp, C.POINTER(ProfileEntry), i32, C.POINTER(C.c_int)]),
    "lc_server_params_default": (None, [C.POINTER(ServerParams)]),
    "lc_server_create": (i32, [C.POINTER(ServerParams), C.POINTER(vp)]),
    "lc_server_destroy": (i32, [vp]),
    "lc_server_submit2d": (i32, [vp, vp, i32, i32, i32, dptr, C.POINTER(C.c_int),
                                 C.POINTER(ReconParamsC), vp, C.POINTER(C.c_longlong)]),
    "lc_server_submit3d": (i32, [vp, vp, i32, i32, i32, dptr, dptr, dptr, vp, C.POINTER(C.c_int),
                                 C.POINTER(ReconParamsC), vp, C.POINTER(C.c_longlong)]),
    "lc_server_wait": (i32, [vp, C.c_longlong, f64, C.POINTER(SolverStats), C.POINTER(JobInfo)]),
    "lc_server_get_stats": (i32, [vp, C.POINTER(ServerStats)]),
    "lc_server_reset_stats": (i32, [vp]),
    "lc_server_clear_psf_cache": (i32, [vp]),
    "lc_server_last_error": (C.c_char_p, [vp]),
}

_lib = None


class LaminocamError(RuntimeError):
    pass


def load(path: str = LIB_PATH):
    """Loads the shared library; raises if it was not built (no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise LaminocamError(
            f"{path} is missing: build it with `python -m laminocam_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
