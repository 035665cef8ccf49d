"""ctypes binding of libdream_das.so (the C ABI in include/dream_das.h).

The library is built in-tree by ``python -m dream_b200.build``. There is no
fallback: if the shared object is missing or fails to load, every entry point
raises, so a CUDA call can never silently run somewhere else.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
# DREAM_DAS_CHECKED=1 selects the bounds-checked build (python -m dream_b200.build --checked)
CHECKED = os.environ.get("DREAM_DAS_CHECKED", "0") not in ("", "0")
LIB_PATH = os.path.join(HERE, "libdream_das_checked.so" if CHECKED else "libdream_das.so")

# status codes (mirror include/dream_das.h)
STATUS_NONE = 0
STATUS_IGNORE_OOB = 1
STATUS_WARN_OOB = 2
STATUS_OOB = 3
ERR_ARGUMENT = -1
ERR_CUDA = -2
ERR_ALLOC = -3
ERR_UNSUPPORTED = -4
ERR_CANCELLED = -5

SAFT, TFM, RCA_COLTX, RCA_ROWTX = 0, 1, 2, 3
LVL_NONE, LVL_IGNORE, LVL_WARN, LVL_STOP = 0, 1, 2, 3
DELAY_SINGLE, DELAY_MULTIPLE = 0, 1
CONV_EQU, CONV_SUM, CONV_NEG = 0, 1, 2
PREC_F64, PREC_F32, PREC_F32_STORE, PREC_BF16_STORE = 0, 1, 2, 3

# every symbol include/dream_das.h declares: name -> (restype, argtypes)
_i, _i64, _d, _vp = ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p
_pi64 = ctypes.POINTER(ctypes.c_int64)
_pd = ctypes.POINTER(ctypes.c_double)
_pp = ctypes.POINTER(ctypes.c_void_p)
SIGNATURES = {
    "dream_das_version": (ctypes.c_char_p, []),
    "dream_das_last_error": (ctypes.c_char_p, []),
    "dream_das_plan_create": (_i, [_pp, _i, _i64, _i64, _i64, _i64, _i, _i]),
    "dream_das_setup_has_changed": (_i, [_vp, _i, _i64, _i64, _i64, _i64, _i, _i]),
    "dream_das_plan_destroy": (None, [_vp]),
    "dream_das_run": (_i, [_vp, _vp, _vp, _vp, _vp, _d, _i, _vp, _d, _vp, _i, _pi64]),
    "dream_das_run_device": (_i, [_vp, _vp, _vp, _vp, _vp, _d, _i, _vp, _d, _vp, _i, _pi64, _vp]),
    "dream_das_run_device_async": (_i, [_vp, _vp, _vp, _vp, _vp, _d, _i, _vp, _d, _vp, _vp, _vp]),
    "dream_das_uni_plan_create": (_i, [_pp, _i, _i64, _pd, _i, _i]),
    "dream_das_plan_num_points": (_i64, [_vp]),
    "dream_das_plan_num_ascans": (_i64, [_vp]),
    "dream_das_plan_launch_count": (_i64, [_vp]),
    "dream_das_checked_build": (ctypes.c_int, []),
    "dream_das_plan_bound_violations": (_i64, [_vp]),
    "dream_das_uni_run": (_i, [_vp, _vp, _pd, _d, _d, _d, _vp, _i, _pi64]),
    "dream_das_uni_run_device": (_i, [_vp, _vp, _pd, _d, _d, _d, _vp, _i, _pi64, _vp]),
    "dream_das_set_grid_hint": (_i, [_vp, _i64]),
    "dream_das_set_tile": (_i, [_vp, _i, _i]),
    "dream_das_set_chunk": (_i, [_vp, _i]),
    "dream_das_set_inner_shard": (_i, [_vp, _i64, _i64]),
    "dream_das_set_l2_block": (_i, [_vp, _i64]),
    "dream_das_indices_device": (_i, [_vp, _vp, _vp, _vp, _d, _i, _vp, _d, _vp, _vp, _vp]),
    "dream_conv_p_run_device": (_i, [_vp, _i64, _i64, _vp, _i64, _i64, _vp, _i, _vp]),
    "dream_conv_p_run": (_i, [_vp, _i64, _i64, _vp, _i64, _i64, _vp, _i, _i]),
    "dream_conv_p_fmc_device": (_i, [_vp, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _vp, _vp]),
    "dream_rect_run_device": (_i, [_vp, _i64, _d, _d, _d, _d, _d, _i64, _i, _vp, _d, _d, _vp, _i, _vp, _i, _vp]),
    "dream_rect_run": (_i, [_vp, _i64, _d, _d, _d, _d, _d, _i64, _i, _vp, _d, _d, _vp, _i, _vp, _i]),
    "dream_arr_rect_run_device": (_i, [_vp, _i64, _d, _d, _d, _d, _d, _i64, _i, _vp, _d, _d, _i64, _vp, _i, _vp,
                                       _i, _d, _d, _i, _vp, _d, _vp, _i, _vp, _i, _vp]),
    "dream_arr_rect_run": (_i, [_vp, _i64, _d, _d, _d, _d, _d, _i64, _i, _vp, _d, _d, _i64, _vp, _i, _vp, _i, _d,
                                _d, _i, _vp, _d, _vp, _i, _vp, _i]),
    "dream_das_get_tile": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "dream_das_weighted_run_device": (_i, [_vp, _vp, _vp, _vp, _vp, _d, _i, _vp, _d, _vp, _vp, _vp, _vp]),
    "dream_das_bind_geometry": (_i, [_vp, _vp, _vp, _vp, _d, _i, _vp, _d, _vp]),
    "dream_das_op_forward": (_i, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "dream_das_op_adjoint": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "dream_das_op_wgrad": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "dream_das_op_backward": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "dream_das_batch_create": (_i, [_pp, _vp, _i, _i, _i]),
    "dream_das_batch_run": (_i, [_vp, _vp, _vp]),
    "dream_das_batch_items": (_i64, [_vp]),
    "dream_das_batch_grid": (_i, [_vp]),
    "dream_das_batch_destroy": (None, [_vp]),
    "dream_das_batch_run_noalloc": (_i, [_vp, _i, _i, _i, _vp, _vp]),
    "dream_das_cancel": (None, [_vp]),
    "dream_das_set_running": (None, [_vp]),
}

_lib = None
_lock = threading.Lock()


class DreamError(RuntimeError):
    """A negative status from the C ABI."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (status {code})")
        self.code = code


def load():
    """Loads libdream_das.so; raises if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is missing: build it with `python -m dream_b200.build"
                    f"{' --checked' if CHECKED else ''}` "
                    "(the CUDA backend has no CPU fallback)")
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def last_error() -> str:
    return load().dream_das_last_error().decode(errors="replace")


def check(code: int) -> int:
    """Raises DreamError for negative status codes; returns the status otherwise."""
    if code < 0:
        raise DreamError(code, last_error() or "DAS error")
    return code


class Plan:
    """Owns a ``dream_das_plan``; destroyed with the object."""

    def __init__(self, handle, key):
        self.handle = handle
        self.key = key

    def __del__(self):
        h, self.handle = getattr(self, "handle", None), None
        if h and _lib is not None:
            _lib.dream_das_plan_destroy(h)

    def cancel(self):
        load().dream_das_cancel(self.handle)

    def set_running(self):
        load().dream_das_set_running(self.handle)


def plan_create(das_type, K, No, Nt, Nr, precision, device=0) -> Plan:
    h = ctypes.c_void_p()
    check(load().dream_das_plan_create(ctypes.byref(h), das_type, K, No, Nt, Nr, precision, device))
    return Plan(h, ("das", das_type, K, No, Nt, Nr, precision, device))


def uni_plan_create(das_type, K, tri, precision, device=0) -> Plan:
    h = ctypes.c_void_p()
    arr = (ctypes.c_double * 15)(*[float(v) for v in tri])
    check(load().dream_das_uni_plan_create(ctypes.byref(h), das_type, K, arr, precision, device))
    return Plan(h, ("uni", das_type, K, tuple(float(v) for v in tri), precision, device))
