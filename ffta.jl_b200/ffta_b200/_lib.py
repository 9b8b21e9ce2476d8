"""ctypes binding of libfftab200.so (the C ABI declared in include/fftab200.h).

The library is built in-tree (``make -C ffta.jl_b200``).  If it is missing
this module raises at import: the package has no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libfftab200.so")

FB_OK = 0
FB_ERR_DIMENSION_MISMATCH = 1
FB_ERR_ARGUMENT = 2
FB_ERR_DOMAIN = 3
FB_ERR_CUDA = 4
FB_ERR_UNSUPPORTED = 5
FB_ERR_OUT_OF_MEMORY = 6

FB_C32 = 0
FB_C64 = 1

# Every symbol include/fftab200.h declares, with its ctypes signature.
_i64 = ctypes.c_int64
_i64p = ctypes.POINTER(ctypes.c_int64)
_vp = ctypes.c_void_p
_plan_p = ctypes.POINTER(ctypes.c_void_p)
SIGNATURES = {
    "fb_plan_create": ([_plan_p, _i64, ctypes.c_int, ctypes.c_int, _i64, _i64, _i64, _i64, _i64,
                        _i64, ctypes.c_uint32], ctypes.c_int),
    "fb_plan_create_2d": ([_plan_p, _i64, _i64, ctypes.c_int, ctypes.c_int, _i64, _i64,
                           ctypes.c_uint32], ctypes.c_int),
    "fb_plan_create_nd": ([_plan_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i64p, _i64p, _i64p,
                           ctypes.c_int, ctypes.POINTER(ctypes.c_int32), _i64, ctypes.c_uint32],
                          ctypes.c_int),
    "fb_plan_create_real": ([_plan_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i64p,
                             ctypes.c_int, ctypes.POINTER(ctypes.c_int32), _i64, ctypes.c_uint32],
                            ctypes.c_int),
    "fb_plan_set_scale": ([_vp, ctypes.c_double], ctypes.c_int),
    "fb_execute": ([_vp, _vp, _vp, _vp], ctypes.c_int),
    "fb_execute_host": ([_vp, _vp, _vp, _vp], ctypes.c_int),
    "fb_execute_batch": ([_vp, _vp, _vp, _i64, _vp], ctypes.c_int),
    "fb_execute_grouped": ([_vp, _i64, ctypes.POINTER(_vp), ctypes.POINTER(_vp), _i64p, _vp],
                           ctypes.c_int),
    "fb_plan_size": ([_vp, ctypes.c_int, _i64p], ctypes.c_int),
    "fb_plan_device_bytes": ([_vp, ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
    "fb_plan_describe": ([_vp, ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
    "fb_plan_destroy": ([_vp], ctypes.c_int),
    "fb_kernel_error_flag": ([ctypes.POINTER(ctypes.c_int), ctypes.c_int], ctypes.c_int),
    "fb_set_wait_limit": ([_i64], ctypes.c_int),
    "fb_execute_noalloc_c32": ([_vp, _vp, _i64, _i64, ctypes.c_int, _vp], ctypes.c_int),
    "fb_server_create": ([_plan_p, ctypes.c_double, ctypes.c_int, ctypes.c_uint32], ctypes.c_int),
    "fb_server_submit": ([_vp, _i64, ctypes.c_int, ctypes.c_int, _i64, _vp, _vp, _i64p],
                         ctypes.c_int),
    "fb_server_submit_many": ([_vp, _i64, _i64p, ctypes.POINTER(ctypes.c_int32),
                               ctypes.POINTER(ctypes.c_int32), _i64p, ctypes.POINTER(_vp),
                               ctypes.POINTER(_vp), _i64p], ctypes.c_int),
    "fb_server_poll": ([_vp, _i64, _i64p, ctypes.POINTER(ctypes.c_double), _i64p], ctypes.c_int),
    "fb_server_wait": ([_vp], ctypes.c_int),
    "fb_server_cancel": ([_vp, _i64], ctypes.c_int),
    "fb_server_drop_next_descriptor": ([_vp], ctypes.c_int),
    "fb_server_stats": ([_vp, _i64p, ctypes.c_int], ctypes.c_int),
    "fb_server_reset_clock": ([_vp], ctypes.c_int),
    "fb_server_destroy": ([_vp], ctypes.c_int),
    "fb_plan_autotune": ([_vp, _vp, _vp, _vp, ctypes.c_int], ctypes.c_int),
    "fb_tune_cache_save": ([ctypes.c_char_p], ctypes.c_int),
    "fb_tune_cache_load": ([ctypes.c_char_p], ctypes.c_int),
    "fb_last_error": ([], ctypes.c_char_p),
    "fb_version": ([], ctypes.c_char_p),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is not built; run `make -C ffta.jl_b200 -j8` (the package has no CPU "
            "fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


lib = _load()


def last_error() -> str:
    return lib.fb_last_error().decode()
