"""ctypes binding of libfvgpu.so (the C ABI declared in include/fvgpu.h).

The shared library is built in-tree for sm_100a (``__graft_entry__.build()`` or
``make -C finitevolumegpu_b200/csrc``).  There is no fallback: if the library
is missing or cannot be loaded, every simulator constructor raises.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfvgpu.so")

FV_OK = 0
FV_ERR_INVALID = 1
FV_ERR_UNSUPPORTED = 2
FV_ERR_CUDA = 3
FV_ERR_DEVICE = 4
FV_ERR_NOMEM = 5

SCHEME_IDS = {
    "LxF": 0,
    "FORCE": 1,
    "HLL": 2,
    "HLL2": 3,
    "WAF": 4,
    "KP07": 5,
    "KP07_dimsplit": 6,
    "EE2D_KP07_dimsplit": 7,
}


class fv_params(ctypes.Structure):
    _fields_ = [
        ("g", ctypes.c_float),
        ("gamma", ctypes.c_float),
        ("theta", ctypes.c_float),
        ("cfl_scale", ctypes.c_float),
        ("order", ctypes.c_int),
        ("tile", ctypes.c_int),
        ("variant", ctypes.c_int),
        ("variant_beta", ctypes.c_float),
    ]


class FVError(RuntimeError):
    """A CUDA or device-side failure reported by libfvgpu."""


_lib = None

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_D = ctypes.c_double
_LL = ctypes.c_longlong
_FP = ctypes.POINTER(ctypes.c_float)

_SIGNATURES = {
    "fv_version": ([], _I),
    "fv_last_error": ([], ctypes.c_char_p),
    "fv_context_create": ([_I, ctypes.POINTER(_P)], _I),
    "fv_context_destroy": ([_P], _I),
    "fv_context_device_name": ([_P, ctypes.c_char_p, _I], _I),
    "fv_sim_create": ([_P, _I, _I, _I, _F, _F, ctypes.POINTER(fv_params), _I, ctypes.POINTER(_FP), _I, _I,
                       ctypes.POINTER(_P)], _I),
    "fv_sim_destroy": ([_P], _I),
    "fv_sim_substep": ([_P, _F, _I], _I),
    "fv_sim_substep_rows": ([_P, _F, _I, _I, _I], _I),
    "fv_sim_tile_rows": ([_P, ctypes.POINTER(_I)], _I),
    "fv_sim_step": ([_P, _F], _I),
    "fv_sim_simulate": ([_P, _D, _F, _I], _I),
    "fv_sim_advance": ([_P, _LL], _I),
    "fv_sim_compute_dt": ([_P, ctypes.POINTER(_F)], _I),
    "fv_sim_download": ([_P, _I, _FP, _I], _I),
    "fv_sim_upload": ([_P, _I, _FP, _I], _I),
    "fv_sim_download_region": ([_P, _I, _I, _I, _I, _I, _FP, _I], _I),
    "fv_sim_upload_region": ([_P, _I, _I, _I, _I, _I, _FP, _I], _I),
    "fv_sim_time": ([_P, ctypes.POINTER(_D), ctypes.POINTER(_LL), ctypes.POINTER(_F)], _I),
    "fv_sim_conservation": ([_P, ctypes.POINTER(_D)], _I),
    "fv_sim_check": ([_P, ctypes.POINTER(_I)], _I),
    "fv_sim_synchronize": ([_P], _I),
    "fv_sim_set_boundary_conditions": ([_P, _I], _I),
    "fv_sim_get_control": ([_P, ctypes.POINTER(_D), ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_float),
                            ctypes.POINTER(ctypes.c_float)], _I),
    "fv_sim_set_control": ([_P, _D, ctypes.c_longlong, ctypes.c_float, ctypes.c_float], _I),
    "fv_sim_buffers": ([_P, ctypes.POINTER(_FP), ctypes.POINTER(_I), ctypes.POINTER(_I)], _I),
    "fv_sim_stream": ([_P, ctypes.POINTER(_P)], _I),
    "fv_sim_info": ([_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)], _I),
    "fv_sim_last_advance_ms": ([_P, ctypes.POINTER(_D)], _I),
    "fv_kp07_dimsplit_substep_noalloc": ([ctypes.POINTER(_FP), ctypes.POINTER(_FP), _I, _I, _I, _F, _F, _F, _F, _F,
                                          _I, _I, _FP, _P], _I),
    "fv_batch_create": ([_P, _I, ctypes.POINTER(fv_params), _I, ctypes.POINTER(_P)], _I),
    "fv_batch_destroy": ([_P], _I),
    "fv_batch_add": ([_P, _I, _I, _F, _F, _I, ctypes.POINTER(_FP), _I, _I, _D, ctypes.POINTER(_I)], _I),
    "fv_batch_remove": ([_P, _I], _I),
    "fv_batch_run": ([_P, _I], _I),
    "fv_batch_sync": ([_P], _I),
    "fv_batch_status": ([_P, _I, ctypes.POINTER(_D), ctypes.POINTER(_LL), ctypes.POINTER(_F), ctypes.POINTER(_I)],
                        _I),
    "fv_batch_download": ([_P, _I, _I, _FP, _I], _I),
    "fv_batch_info": ([_P, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(_I), ctypes.POINTER(_I),
                       ctypes.POINTER(_D)], _I),
    "fv_batch_tile": ([_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)], _I),
    "fv_sim_set_wait_limit": ([_P, _I], _I),
    "fv_selftest_bounded_wait": ([_I, ctypes.POINTER(_I)], _I),
    "fv_host_alloc": ([ctypes.POINTER(_P), ctypes.c_size_t], _I),
    "fv_host_free": ([_P], _I),
}


def lib():
    """Load libfvgpu.so once; raise if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                "libfvgpu.so is not built (expected at %s); build it with "
                "`make -C finitevolumegpu_b200/csrc` or __graft_entry__.build()" % LIB_PATH
            )
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def require(cond, msg="invalid argument") -> None:
    """An argument check that raises the reference's AssertionError and, unlike
    an assert statement, still runs under ``python -O``: it guards the sizes of
    host buffers handed to the C library."""
    if not cond:
        raise AssertionError(msg)


def check(rc: int) -> None:
    """Map a C status code to the reference's Python exception types."""
    if rc == FV_OK:
        return
    msg = lib().fv_last_error().decode(errors="replace")
    if rc == FV_ERR_INVALID:
        raise AssertionError(msg)
    if rc == FV_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    if rc == FV_ERR_NOMEM:
        raise MemoryError(msg)
    raise FVError(msg)
