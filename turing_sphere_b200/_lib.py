"""ctypes binding of libturing_sht.so (declared in include/turing_sht.h).

This module is the Python counterpart of the N-API/koffi binding a TypeScript
host would use; it passes only plain pointers, sizes and ints.  There is no
fallback: if the shared library is missing the import fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libturing_sht.so")

TS_OK = 0
TS_ERR_INVALID = -1
TS_ERR_CUDA = -2
TS_ERR_COMPILE = -3
TS_ERR_NOT_FOUND = -4
TS_ERR_SIZE = -5
TS_ERR_UNSUPPORTED = -6
TS_ERR_TIMEOUT = -7
TS_ERR_STATE = -8

TS_PREC_FP32 = 0
TS_PREC_TF32X3 = 1
TS_PREC_BF16X3 = 2
TS_FOURIER_AUTO = 0
TS_FOURIER_FFT = 0x10
TS_FOURIER_DFT = 0x20
TS_PLAN_AUTOTUNE = 0x40
TS_CHECK_SOURCE = 0x100
TS_CHECK_ADJOINT = 0x200

STATUS_NAMES = {
    TS_ERR_INVALID: "invalid", TS_ERR_CUDA: "cuda", TS_ERR_COMPILE: "compile",
    TS_ERR_NOT_FOUND: "not_found", TS_ERR_SIZE: "size", TS_ERR_UNSUPPORTED: "unsupported",
    TS_ERR_TIMEOUT: "timeout", TS_ERR_STATE: "state",
}


class TsError(RuntimeError):
    """A failed C-ABI call: ``status`` is the ts_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class PlanInfo(C.Structure):
    _fields_ = [
        ("lmax", C.c_int), ("mmax", C.c_int), ("nlat", C.c_int), ("nphi", C.c_int),
        ("nlm", C.c_long), ("precision", C.c_int), ("fourier", C.c_int),
        ("fft_stages", C.c_int), ("fft_radix", C.c_int * 16), ("table_bytes", C.c_long),
        ("tc_lat_tile", C.c_int), ("tc_deg_tile", C.c_int), ("fft_p", C.c_int),
        ("fft_q", C.c_int), ("fft_rows", C.c_int), ("tuned", C.c_int),
        ("tc_skip_tiles", C.c_int), ("tc_skip_chunks", C.c_int),
    ]


class CompileError(C.Structure):
    _fields_ = [("start", C.c_long), ("end", C.c_long), ("fn", C.c_char * 64),
                ("message", C.c_char * 1024)]


vp = C.c_void_p
i32 = C.c_int
i64 = C.c_long
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
cstr = C.c_char_p

# name -> (restype, argtypes); every symbol declared in include/turing_sht.h
SIGNATURES = {
    "ts_ctx_create": (i32, [i32, C.POINTER(vp)]),
    "ts_ctx_destroy": (i32, [vp]),
    "ts_last_error": (cstr, [vp]),
    "ts_ctx_set_stream": (i32, [vp, vp]),
    "ts_ctx_stream": (vp, [vp]),
    "ts_ctx_device_name": (i32, [vp, C.c_char_p, C.c_size_t]),
    "ts_sync": (i32, [vp]),
    "ts_nlm_calc": (i64, [i32, i32]),
    "ts_lm_index": (i64, [i32, i32, i32]),
    "ts_validate_config": (i32, [i32, i32, i32, i32, C.c_char_p, C.c_size_t]),
    "ts_grid_for_lmax": (None, [i32, i32, C.POINTER(i32), C.POINTER(i32)]),
    "ts_sht_plan_create": (i32, [vp, i32, i32, i32, i32, i32, C.POINTER(vp)]),
    "ts_sht_plan_destroy": (i32, [vp]),
    "ts_sht_plan_info": (i32, [vp, C.POINTER(PlanInfo)]),
    "ts_sht_plan_nodes": (i32, [vp, f64p, f64p]),
    "ts_sht_plan_status": (i32, [vp]),
    "ts_sht_synth_dev": (i32, [vp, vp, vp, i32, vp]),
    "ts_sht_analys_dev": (i32, [vp, vp, vp, i32, vp]),
    "ts_sht_synth_noalloc": (i32, [vp, vp, vp, i32, vp]),
    "ts_sht_synth": (i32, [vp, f32p, i64, f32p, i64, i32]),
    "ts_sht_analys": (i32, [vp, f32p, i64, f32p, i64, i32]),
    "ts_sht_roundtrip": (i32, [vp, vp, i64, vp, i64, i32]),
    "ts_sht_leg_synth_dev": (i32, [vp, vp, vp, i32, vp]),
    "ts_sht_fourier_synth_dev": (i32, [vp, vp, vp, i32, vp]),
    "ts_sht_fourier_analys_dev": (i32, [vp, vp, vp, i32, vp]),
    "ts_sht_leg_analys_dev": (i32, [vp, vp, vp, i32, vp]),
    "ts_sht_wimage_bytes": (C.c_size_t, [vp, i32]),
    "ts_sht_plan_test_stall": (i32, [vp, i32, C.c_uint]),
    "ts_sht_synth_adjoint_dev": (i32, [vp, vp, vp, i32, vp]),
    "ts_sht_analys_adjoint_dev": (i32, [vp, vp, vp, i32, vp]),
    "ts_sht_fourier_analys_w_dev": (i32, [vp, vp, vp, i32, vp]),
    "ts_sht_leg_analys_w_dev": (i32, [vp, vp, vp, i32, vp]),
    "ts_model_compile": (i32, [vp, cstr, C.POINTER(cstr), i32, C.POINTER(cstr), i32,
                               C.POINTER(cstr), i32, i32, C.POINTER(vp), C.POINTER(CompileError)]),
    "ts_model_destroy": (i32, [vp]),
    "ts_model_set_params": (i32, [vp, f32p, i32]),
    "ts_model_set_params_batched": (i32, [vp, f32p, i32, i32]),
    "ts_model_upload": (i32, [vp, cstr, f32p, i64]),
    "ts_model_init": (i32, [vp, f32p, i64]),
    "ts_model_step": (i32, [vp, i32]),
    "ts_model_set_graphs": (i32, [vp, i32]),
    "ts_model_forward_backward": (i32, [vp, i32, i32, f32p, f32p, f64p]),
    "ts_model_group_create": (i32, [C.POINTER(vp), i32, C.POINTER(vp)]),
    "ts_model_group_step": (i32, [vp, i32]),
    "ts_model_group_destroy": (i32, [vp]),
    "ts_model_read": (i32, [vp, cstr, f32p, i64]),
    "ts_model_value_ptr": (i32, [vp, cstr, C.POINTER(vp), C.POINTER(i64)]),
    "ts_model_snapshot": (i32, [vp]),
    "ts_model_restore": (i32, [vp]),
    "ts_model_describe": (i32, [vp, i32, C.c_char_p, C.c_size_t]),
    "ts_model_source": (i32, [vp, C.c_char_p, C.c_size_t]),
    "ts_model_counts": (i32, [vp, i32, C.POINTER(i32), C.POINTER(i32)]),
    "ts_model_check": (i32, [i32, i32, i32, i32, cstr, C.POINTER(cstr), i32, C.POINTER(cstr), i32,
                             C.POINTER(cstr), i32, i32, i32, C.c_char_p, C.c_size_t, C.POINTER(i32),
                             C.POINTER(i32), C.POINTER(CompileError)]),
    "ts_seeded_noise": (None, [i64, C.c_double, C.c_uint, f32p]),
    "ts_seeded_spectrum": (None, [i32, i32, C.c_uint, f32p]),
}

_lib = None


def lib():
    """Load the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C turing_sphere_b200/csrc` "
                "(or __graft_entry__.build()); there is no non-CUDA fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, ctx=None) -> None:
    if status != TS_OK:
        msg = lib().ts_last_error(ctx)
        raise TsError(status, (msg or b"").decode() or STATUS_NAMES.get(status, str(status)))


def cstr_array(names):
    arr = (cstr * max(1, len(names)))()
    for i, n in enumerate(names):
        arr[i] = n.encode()
    return arr


def fptr(a):
    """float* of a C-contiguous float32 numpy array."""
    return a.ctypes.data_as(f32p)


def dptr(a):
    return a.ctypes.data_as(f64p)
