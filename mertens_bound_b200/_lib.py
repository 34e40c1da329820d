"""ctypes binding of libmertens_k2.so (declared in include/mertens_k2.h).

The library is built in-tree (python -m mertens_bound_b200.build).  There is no CPU
fallback: if the library is missing or cannot be loaded, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmertens_k2.so")

u64p = C.POINTER(C.c_uint64)
f64p = C.POINTER(C.c_double)
i64p = C.POINTER(C.c_int64)
vp = C.c_void_p
i64 = C.c_int64
f64 = C.c_double
i32 = C.c_int

# name -> (restype, argtypes); every function declared in include/mertens_k2.h appears here.
SIGNATURES: dict[str, tuple] = {
    "mb_last_error": (C.c_char_p, []),
    "mb_abi_version": (i32, []),
    "mb_table_create": (i32, [vp, vp, vp, vp, i64, i32, C.POINTER(vp)]),
    "mb_table_destroy": (i32, [vp]),
    "mb_table_size": (i32, [vp, i64p]),
    "mb_table_count_below": (i32, [vp, f64, i64p]),
    "mb_phase128": (i32, [vp, i64, vp, vp, i64, vp, vp]),
    "mb_k2_plain": (i32, [vp, i64, vp, vp, vp, f64, f64, vp, vp, vp]),
    "mb_k2_plain_dev": (i32, [vp, i64, vp, vp, vp, f64, f64, vp, vp, vp, vp]),
    "mb_plan_create": (i32, [vp, i32, vp, vp, vp, f64, C.POINTER(vp)]),
    "mb_plan_destroy": (i32, [vp]),
    "mb_table_add_weights": (i32, [vp, vp, i64, C.POINTER(i32)]),
    "mb_plan_create_weighted": (i32, [vp, i32, vp, vp, vp, vp, f64, C.POINTER(vp)]),
    "mb_plan_set_skip": (i32, [vp, f64]),
    "mb_plan_group_zeros": (i32, [vp, i32, i64p]),
    "mb_plan_group_bounds": (i32, [vp, i32, f64p, f64p, f64p]),
    "mb_plan_autotune": (i32, [vp, i32, C.POINTER(i32), C.POINTER(i32), f64p, f64p, f64p]),
    "mb_plan_set_shape": (i32, [vp, i32, i32, i32, i64, i64]),
    "mb_plan_info": (i32, [vp, i64p, f64p, C.POINTER(i32)]),
    "mb_plan_light_form": (i32, [vp, C.POINTER(i32)]),
    "mb_plan_configure": (i32, [vp, i32, i32, f64]),
    "mb_plan_set_schedule": (i32, [vp, i32]),
    "mb_plan_schedule": (i32, [vp, C.POINTER(i32)]),
    "mb_plan_set_zero_range": (i32, [vp, i64, i64]),
    "mb_plan_time": (i32, [vp, i32, f64p]),
    "mb_plan_group_info": (i32, [vp, i32, i64p, i64p, f64p, f64p]),
    "mb_plan_run_dev": (i32, [vp, vp, vp, vp, vp, vp, vp, vp]),
    "mb_plan_run": (i32, [vp, vp, vp, vp, vp, vp, vp]),
    "mb_k2_fast": (i32, [vp, i64, vp, vp, vp, f64, f64, f64, vp, vp, vp, f64p]),
    "mb_plan_run_tiers_dev": (i32, [vp, i32, vp, vp, vp, vp, vp, vp, vp]),
    "mb_plan_newton_dev": (i32, [vp, vp, vp, vp, i32, f64, vp, vp, vp, vp, vp]),
    "mb_plan_tier_terms": (i32, [vp, f64p, f64p]),
    "mb_calibrate_issue": (i32, [i32, f64p]),
    "mb_calibrate_pipes": (i32, [i32, f64p, f64p, f64p]),
    "mb_plan_kernel_timing": (i32, [vp, i32]),
    "mb_plan_kernel_times": (i32, [vp, i32, vp, vp, C.POINTER(i32)]),
    "mb_k2_plain_noalloc_dev": (i32, [vp, vp, vp, vp, i64, i64, i64, vp, vp, vp, f64, vp, vp, vp, vp]),
    "mb_k2_certified": (i32, [vp, i64, vp, vp, vp, f64, f64, vp, vp, vp, vp]),
    "mb_k2_certified_range": (i32, [vp, i64, vp, vp, vp, f64, f64, i64, i64, vp, vp, vp, vp]),
    "mb_k2_certified_grad_range": (i32, [vp, i64, vp, vp, vp, f64, f64, i64, i64, vp, vp, vp]),
    "mb_grid_scan": (i32, [vp, i64, vp, vp, f64, f64, C.c_uint64, C.c_uint64, i64, i64, vp]),
    "mb_hit_scan": (i32, [vp, i64, vp, vp, f64, i64, C.c_uint64, C.c_uint64, i64, i64, vp]),
    "mb_exact_AB": (i32, [vp, i64, vp, vp, vp, i64, vp, vp]),
    "mb_polish_single_peak": (i32, [i64, i64, i64, vp, vp, vp, vp, f64, i32, vp, vp, vp]),
    "mb_fast_polish_batch": (i32, [i64, i64, vp, vp, vp, vp, vp, i64, i32, vp, vp, vp]),
    "mb_polish_single_exact": (i32, [vp, i64, vp, vp, vp, i64, i32, f64, i32, vp, vp, vp]),
    "mb_polish_peaks_exact": (i32, [vp, i64, vp, vp, vp, i64, i32, f64, i32, vp, vp, vp]),
    "mb_polish_peaks_weights": (i32, [vp, i64, vp, vp, vp, i64, i32, vp, f64, i32, vp, vp, vp]),
    "mb_fast_polish_exact": (i32, [vp, i64, vp, vp, vp, i64, i32, vp, i64, i32, vp, vp, vp]),
    "mb_screen": (i32, [vp, i64, vp, vp, f64, C.c_uint64, C.c_uint64, i32, vp, vp, i64, vp, vp, vp, vp]),
    "mb_screen_dev": (i32, [vp, i64, vp, vp, f64, C.c_uint64, C.c_uint64, i32, vp, vp, i64, vp, vp, vp, vp, vp]),
    "compute_peak_AB": (None, [i32, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "polish_peaks_with_weights": (None, [i32, i32, vp, vp, vp, vp, f64, i32, vp, vp, vp]),
    "mb_compute_peak_AB": (i32, [i32, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "mb_polish_peaks_with_weights": (i32, [i32, i32, vp, vp, vp, vp, f64, i32, vp, vp, vp]),
}


class K2Error(RuntimeError):
    """A libmertens_k2 call returned a nonzero status."""

    NAMES = {-1: "MB_ERR_ARG", -2: "MB_ERR_TABLE", -3: "MB_ERR_CUDA", -4: "MB_ERR_TIMEOUT",
             -5: "MB_ERR_STATE", -6: "MB_ERR_CAPACITY"}

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{self.NAMES.get(status, status)}: {message}")


_lock = threading.Lock()
_lib = None


def lib():
    """The loaded library (loaded once; raises if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(f"{LIB_PATH} is not built; run python -m mertens_bound_b200.build")
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def check(status: int) -> None:
    if status != 0:
        msg = lib().mb_last_error()
        raise K2Error(status, msg.decode() if msg else "")


def ptr(a) -> int:
    """Data pointer of a contiguous numpy array (or None)."""
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data
