"""ctypes binding of libthistle_b200.so (declared in include/thistle_b200.h).

The library is built in-tree by ``thistle_b200.build``; importing this module
without it raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# THISTLE_B200_LIB selects another build of the same library (e.g. a tuning variant)
LIB_PATH = os.environ.get("THISTLE_B200_LIB") or os.path.join(_HERE, "libthistle_b200.so")

ERRORS = {
    -1: "THISTLE_ERR_ARG", -2: "THISTLE_ERR_SHAPE", -3: "THISTLE_ERR_ANGMOM", -4: "THISTLE_ERR_NONFINITE",
    -5: "THISTLE_ERR_CUDA", -6: "THISTLE_ERR_NOMEM", -7: "THISTLE_ERR_TYPE", -8: "THISTLE_ERR_Q",
}

# every symbol include/thistle_b200.h declares
EXPORTS = sorted([
    "thistle_last_error_string", "thistle_version", "thistle_total_scattering", "thistle_probe_fp64_peak",
    "thistle_plan_create", "thistle_plan_set_stream", "thistle_plan_set_centres", "thistle_plan_execute",
    "thistle_plan_execute_device", "thistle_plan_recompute_device", "thistle_plan_execute_quartets",
    "thistle_plan_info", "thistle_plan_class_counts", "thistle_plan_timings", "thistle_plan_stage_totals",
    "thistle_plan_destroy", "thistle_plan_records", "thistle_bessel_sum_static",
    "thistle_release_device_cache", "thistle_device_cache_bytes", "thistle_plan_execute_aligned",
    "thistle_qcoord3", "thistle_plan_vjp", "thistle_plan_vjp_device", "thistle_plan_set_batch",
    "thistle_plan_set_centres_batch", "thistle_plan_execute_batch", "thistle_plan_execute_batch_device",
    "thistle_plan_vjp_batch", "thistle_plan_vjp_batch_device", "thistle_plan_use_graph",
    "thistle_plan_autotune_batch", "thistle_batch_create", "thistle_batch_use_graph", "thistle_batch_execute",
    "thistle_batch_execute_device", "thistle_batch_info", "thistle_batch_destroy", "thistle_plan_nuclear",
    "thistle_plan_density", "thistle_plan_form_factor", "thistle_elastic_aligned_grid",
    "thistle_plan_set_centres_batch_device", "thistle_plan_set_stage2_tile", "thistle_plan_stage2_tile",
    "thistle_batch_set_stage2_tile", "thistle_batch_stage2_tile", "thistle_batch_autotune",
    "thistle_plan_set_pipeline",
])


class ThistleError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None

D = C.POINTER(C.c_double)
I32 = C.POINTER(C.c_int32)
I64 = C.POINTER(C.c_int64)
VP = C.c_void_p


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ThistleError(-5, f"CUDA extension not built: {LIB_PATH} is missing (run python -m thistle_b200.build)")
    L = C.CDLL(LIB_PATH)
    L.thistle_last_error_string.restype = C.c_char_p
    L.thistle_last_error_string.argtypes = []
    L.thistle_version.restype = C.c_int
    L.thistle_total_scattering.restype = C.c_int
    L.thistle_total_scattering.argtypes = [
        C.c_int32, D, D, C.c_int32, C.c_int32, C.c_int32, C.c_int32, D, I32, I32, I32, D, D, D, D, C.c_int32,
        D, C.c_int32, I32, C.c_double, C.c_double, C.c_double, I32, D, C.c_int32, D, C.c_int32, D, D]
    L.thistle_plan_create.restype = C.c_int
    L.thistle_plan_create.argtypes = [
        C.POINTER(VP), C.c_int32, C.c_int32, D, I32, I32, I32, D, D, D, I32, D, C.c_int32, I32, D, C.c_int32,
        D, C.c_int32, D, C.c_int32, C.c_double, C.c_double, C.c_double]
    L.thistle_probe_fp64_peak.restype = C.c_int
    L.thistle_probe_fp64_peak.argtypes = [C.c_int32, D]
    L.thistle_plan_set_stream.restype = C.c_int
    L.thistle_plan_set_stream.argtypes = [VP, VP]
    L.thistle_plan_recompute_device.restype = C.c_int
    L.thistle_plan_recompute_device.argtypes = [VP, VP]
    L.thistle_plan_class_counts.restype = C.c_int
    L.thistle_plan_class_counts.argtypes = [VP, I64]
    L.thistle_plan_stage_totals.restype = C.c_int
    L.thistle_plan_stage_totals.argtypes = [VP, D, I64]
    L.thistle_plan_records.restype = C.c_int
    L.thistle_plan_records.argtypes = [VP, C.POINTER(VP), I32, I64, I64, I64, I32, C.POINTER(VP)]
    L.thistle_bessel_sum_static.restype = C.c_int
    L.thistle_bessel_sum_static.argtypes = [VP, C.c_int32, I64, I64, I64, I32, VP, C.c_int32, VP, VP]
    L.thistle_plan_set_centres.restype = C.c_int
    L.thistle_plan_set_centres.argtypes = [VP, D, D, D]
    L.thistle_plan_execute.restype = C.c_int
    L.thistle_plan_execute.argtypes = [VP, D]
    L.thistle_plan_execute_device.restype = C.c_int
    L.thistle_plan_execute_device.argtypes = [VP, VP]
    L.thistle_plan_execute_quartets.restype = C.c_int
    L.thistle_plan_execute_quartets.argtypes = [VP, I32, C.c_int64, D]
    L.thistle_plan_info.restype = C.c_int
    L.thistle_plan_info.argtypes = [VP, I64]
    L.thistle_plan_timings.restype = C.c_int
    L.thistle_plan_timings.argtypes = [VP, D]
    L.thistle_plan_destroy.restype = C.c_int
    L.thistle_plan_destroy.argtypes = [VP]
    L.thistle_plan_execute_aligned.restype = C.c_int
    L.thistle_plan_execute_aligned.argtypes = [VP, D, D]
    L.thistle_plan_vjp.restype = C.c_int
    L.thistle_plan_vjp.argtypes = [VP, D, D]
    L.thistle_plan_vjp_device.restype = C.c_int
    L.thistle_plan_vjp_device.argtypes = [VP, VP, VP]
    for name, args in (("thistle_plan_set_batch", [VP, C.c_int32]), ("thistle_plan_set_centres_batch", [VP, D]),
                       ("thistle_plan_execute_batch", [VP, D]), ("thistle_plan_execute_batch_device", [VP, VP]),
                       ("thistle_plan_vjp_batch", [VP, D, D]), ("thistle_plan_vjp_batch_device", [VP, VP, VP]),
                       ("thistle_plan_use_graph", [VP, C.c_int32]),
                       ("thistle_plan_autotune_batch", [VP, C.c_int32, I32, I32, D]),
                       ("thistle_batch_create", [C.POINTER(VP), C.POINTER(VP), C.c_int32]),
                       ("thistle_batch_use_graph", [VP, C.c_int32]), ("thistle_batch_execute", [VP, D]),
                       ("thistle_batch_execute_device", [VP, VP]), ("thistle_batch_info", [VP, I64]),
                       ("thistle_batch_destroy", [VP]), ("thistle_plan_nuclear", [VP, D, D, C.c_int32, D]),
                       ("thistle_plan_set_stage2_tile", [VP, C.c_int32, C.c_int32]),
                       ("thistle_plan_set_pipeline", [VP, C.c_int32]),
                       ("thistle_plan_stage2_tile", [VP, I32, I32]),
                       ("thistle_batch_set_stage2_tile", [VP, C.c_int32, C.c_int32]),
                       ("thistle_batch_stage2_tile", [VP, I32, I32]),
                       ("thistle_batch_autotune", [VP, I32, I32, D])):
        getattr(L, name).restype = C.c_int
        getattr(L, name).argtypes = args
    L.thistle_qcoord3.restype = C.c_int
    L.thistle_qcoord3.argtypes = [C.c_double, D]
    L.thistle_release_device_cache.restype = C.c_int
    L.thistle_release_device_cache.argtypes = []
    L.thistle_device_cache_bytes.restype = C.c_int
    L.thistle_device_cache_bytes.argtypes = [I64, I64]
    _lib = L
    return L


def device_cache_bytes():
    """(cached, in_use) bytes of the library's device-buffer cache on the current device."""
    c, u = C.c_int64(0), C.c_int64(0)
    check(lib().thistle_device_cache_bytes(C.byref(c), C.byref(u)))
    return c.value, u.value


def release_device_cache():
    """Return the cached device buffers and idle cuBLAS handles of the current device to the driver."""
    check(lib().thistle_release_device_cache())


def check(rc: int):
    if rc != 0:
        msg = lib().thistle_last_error_string()
        raise ThistleError(rc, msg.decode() if msg else "")


def dptr(a):
    return None if a is None else a.ctypes.data_as(D)


def iptr(a):
    return None if a is None else a.ctypes.data_as(I32)


def as_f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def as_i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


def colmajor_f64(a):
    """Fortran-order flat copy of a 2-D array."""
    return None if a is None else np.ascontiguousarray(np.asarray(a, dtype=np.float64).T)


def colmajor_i32(a):
    return None if a is None else np.ascontiguousarray(np.asarray(a, dtype=np.int32).T)
