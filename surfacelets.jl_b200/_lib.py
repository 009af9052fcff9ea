"""ctypes binding of libsurfacelets_b200.so (include/surfacelets_b200.h).

The library is loaded from this directory.  A missing library raises at
import time: there is no CPU fallback behind this package.
"""

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsurfacelets_b200.so")

SFL_OK = 0
SFL_DONE = 1
SFL_ERR_ARGUMENT = -1
SFL_ERR_DIMENSION = -2
SFL_ERR_CUDA = -3
SFL_ERR_ALLOC = -4
SFL_ERR_STATE = -5
SFL_ERR_UNSUPPORTED = -6
SFL_ERR_TIMEOUT = -7
SFL_MAX_SCALES = 16
SFL_REAL32 = 0
SFL_COMPLEX64 = 1
SFL_KIND_NS = 0
SFL_KIND_DECIMATED = 1


class NSParams(C.Structure):
    _fields_ = [
        ("scales", C.c_int32),
        ("direction_levels", C.c_int32 * SFL_MAX_SCALES),
        ("bernstein_order", C.c_int32),
        ("halfband_order", C.c_int32),
        ("transition", C.c_double),
        ("tight", C.c_int32),
    ]


class SurfParams(C.Structure):
    _fields_ = [
        ("scales", C.c_int32),
        ("levels", ((C.c_int32 * 3) * 3) * SFL_MAX_SCALES),
        ("pyramid_ratio", C.c_double),
        ("checkerboard_order", C.c_int32),
        ("diamond_length", C.c_int32),
        ("kaiser_beta", C.c_double),
        ("diamond_power", C.c_int32),
    ]


class NDFBParams(C.Structure):
    """sfl_ndfb_params"""
    _fields_ = [
        ("levels", C.c_int32),
        ("bernstein_order", C.c_int32),
        ("halfband_order", C.c_int32),
        ("transition", C.c_double),
        ("tight", C.c_int32),
    ]


Dims = C.c_int32 * 3
P = C.c_void_p

# name -> (restype, argtypes)
SIGNATURES = {
    "sfl_last_error": (C.c_char_p, []),
    "sfl_version": (C.c_char_p, []),
    "sfl_ns_check_params": (C.c_int, [C.POINTER(NSParams)]),
    "sfl_ns_check_size": (C.c_int, [C.POINTER(NSParams), Dims]),
    "sfl_ns_nsubbands": (C.c_int, [C.POINTER(NSParams), C.POINTER(C.c_int32)]),
    "sfl_ns_layout": (C.c_int, [C.POINTER(NSParams), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "sfl_surf_levels_from_int": (C.c_int, [C.c_int32, (C.c_int32 * 3) * 3]),
    "sfl_surf_check_params": (C.c_int, [C.POINTER(SurfParams)]),
    "sfl_surf_layout": (C.c_int, [C.POINTER(SurfParams), Dims, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                  C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "sfl_surf_redundancy": (C.c_int, [C.POINTER(SurfParams), Dims, C.POINTER(C.c_double)]),
    "sfl_ns_plan_create": (C.c_int, [C.POINTER(NSParams), Dims, C.c_int32, C.POINTER(P)]),
    "sfl_ndfb_check_params": (C.c_int, [C.POINTER(NDFBParams)]),
    "sfl_ndfb_plan_create": (C.c_int, [C.POINTER(NDFBParams), Dims, C.c_int32, C.POINTER(P)]),
    "sfl_surf_plan_create": (C.c_int, [C.POINTER(SurfParams), Dims, C.c_int32, C.POINTER(P)]),
    "sfl_plan_destroy": (C.c_int, [P]),
    "sfl_plan_info": (C.c_int, [P, C.POINTER(C.c_int32), Dims, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                C.POINTER(C.c_int64)]),
    "sfl_subband_info": (C.c_int, [P, C.c_int32, Dims, C.POINTER(C.c_int64)]),
    "sfl_plan_set_group": (C.c_int, [P, C.c_int32]),
    "sfl_plan_set_pipeline": (C.c_int, [P, C.c_int32]),
    "sfl_plan_tuning": (C.c_int, [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "sfl_plan_autotune": (C.c_int, [P, P, P, P]),
    "sfl_plan_status": (C.c_int, [P, C.POINTER(C.c_int32), C.c_int32]),
    "sfl_plan_selftest_wait": (C.c_int, [P, P]),
    "sfl_plan_tile": (C.c_int, [P, C.c_int32, C.POINTER(C.c_int32)]),
    "sfl_analyze": (C.c_int, [P, P, P, P]),
    "sfl_synthesize": (C.c_int, [P, P, P, P]),
    "sfl_adjoint_analyze": (C.c_int, [P, P, P, P]),
    "sfl_adjoint_synthesize": (C.c_int, [P, P, P, P]),
    "sfl_stream_analyze_begin": (C.c_int, [P, P, P]),
    "sfl_stream_analyze_next": (C.c_int, [P, P, C.POINTER(C.c_int32), P]),
    "sfl_stream_synthesize_begin": (C.c_int, [P, P]),
    "sfl_stream_synthesize_next_index": (C.c_int, [P, C.POINTER(C.c_int32)]),
    "sfl_stream_synthesize_push": (C.c_int, [P, P, P]),
    "sfl_stream_synthesize_end": (C.c_int, [P, P, P]),
    "sfl_ns_analyze_subband_static": (C.c_int, [P, P, P, C.c_int32, P]),
    "sfl_ns_design_table": (C.c_int, [C.POINTER(NSParams), Dims, C.c_char_p, C.c_int32,
                                      C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "sfl_surf_design_table": (C.c_int, [C.POINTER(SurfParams), Dims, C.c_char_p, C.c_int32,
                                        C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "sfl_ns_plan_table": (C.c_int, [P, C.c_char_p, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_int64)]),
    "sfl_surf_plan_table": (C.c_int, [P, C.c_char_p, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_int64)]),
    "sfl_ns_denoise": (C.c_int, [P, P, P, P, P]),
    "sfl_ns_spectrum_elems": (C.c_int, [P, C.POINTER(C.c_int64)]),
    "sfl_ns_stream_order": (C.c_int, [P, C.POINTER(C.c_int32)]),
    "sfl_ns_forward_spectrum": (C.c_int, [P, P, P, P]),
    "sfl_ns_analyze_range": (C.c_int, [P, P, C.c_int32, C.c_int32, P, P]),
    "sfl_ns_accumulate_range": (C.c_int, [P, P, C.c_int32, C.c_int32, P, C.c_int32, P]),
    "sfl_ns_inverse_spectrum": (C.c_int, [P, P, P, P]),
    "sfl_ns_analyze_bf16": (C.c_int, [P, P, P, P, P]),
    "sfl_ns_synthesize_bf16": (C.c_int, [P, P, P, P, P]),
    "sfl_batch_create": (C.c_int, [C.c_int32, C.POINTER(P), C.POINTER(C.c_int32), C.POINTER(P), C.POINTER(P),
                                   C.POINTER(P)]),
    "sfl_batch_run": (C.c_int, [P, P]),
    "sfl_batch_destroy": (C.c_int, [P]),
    "sfl_profile_enable": (C.c_int, [C.c_int32]),
    "sfl_profile_reset": (C.c_int, []),
    "sfl_profile_read": (C.c_int, [C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "sfl_profile_tags": (C.c_int, [C.c_char_p, C.c_int64]),
    "sfl_profile_bytes": (C.c_int, [C.c_char_p, C.POINTER(C.c_double)]),
}


class ArgumentError(ValueError):
    """The reference's ArgumentError."""


class DimensionMismatch(ValueError):
    """The reference's DimensionMismatch."""


class CudaError(RuntimeError):
    pass


class StateError(RuntimeError):
    pass


class DeviceWaitTimeout(RuntimeError):
    """A bounded device wait of an earlier call on the plan ran out; that
    call's results are not valid (reported once by the next call)."""


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python surfacelets.jl_b200/build.py` "
            "(the package has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status):
    """Raise the exception that a status code stands for."""
    if status >= 0:
        return status
    msg = lib.sfl_last_error().decode("utf-8", "replace")
    if status == SFL_ERR_ARGUMENT:
        raise ArgumentError(msg)
    if status == SFL_ERR_DIMENSION:
        raise DimensionMismatch(msg)
    if status == SFL_ERR_STATE:
        raise StateError(msg)
    if status == SFL_ERR_ALLOC:
        raise MemoryError(msg)
    if status == SFL_ERR_TIMEOUT:
        raise DeviceWaitTimeout(msg)
    raise CudaError(msg)
