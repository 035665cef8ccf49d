"""DREAM's DAS call surface on the CUDA backend.

``das(Y, Gt, Gr, Ro, dt, delay, cp, method, err_level, device, verbose)``
keeps the argument order, shapes, method and error-level strings, and error
behaviour of the reference Python binding (python/src/py_das.cc:40-88,
python/include/py_das.hpp:34-247); ``das_uni`` mirrors the Octave
``das_uni`` (extra_src/oct_das_uni.cc:43-495). The device string selects the
backend: ``'cuda'`` (or ``'cuda:N'``; ``'gpu'`` is accepted as an alias)
runs the sm_100a kernels of libdream_das.so. ``'cpu'`` stays with the
reference's own module -- this package has no CPU implementation and never
falls back to one.

Inputs may be NumPy arrays (host; the call copies through the C ABI's host
entry point, like a reference binding would) or torch tensors on a CUDA
device (no host round trip; the result stays on the device).
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np

from . import _lib

_METHODS = {"saft": _lib.SAFT, "tfm": _lib.TFM, "rca": _lib.RCA_COLTX,
            "rca_coltx": _lib.RCA_COLTX, "rca_rowtx": _lib.RCA_ROWTX}
_LEVELS = {"ignore": _lib.LVL_IGNORE, "warn": _lib.LVL_WARN, "stop": _lib.LVL_STOP}

# Per-thread cached plans: the analogue of the module-global DAS object the
# reference binding keeps (python/src/py_das.cc:30-34), reused while the setup
# is unchanged (include/das.h:77-94).
_tls = threading.local()


def parse_method(method: str) -> int:
    """``parse_das_arg`` (include/arg_parser_python.h:552-592)."""
    if method not in _METHODS:
        raise RuntimeError("Error in das!")  # 'das Unknown delay-and-sum method!'
    return _METHODS[method]


def parse_err_level(err_level: str) -> int:
    """``parse_error_arg`` (include/arg_parser_python.h:277-300)."""
    if err_level not in _LEVELS:
        raise RuntimeError("Error in das!")  # 'das Unknown error level!'
    return _LEVELS[err_level]


def parse_device(device: str) -> int:
    """'cuda', 'cuda:N' or 'gpu' -> CUDA ordinal. 'cpu' is the reference's."""
    d = str(device)
    if d in ("cuda", "gpu"):
        return 0
    if d.startswith("cuda:") and d[5:].isdigit():
        return int(d[5:])
    if d == "cpu":
        raise RuntimeError(
            "das: device 'cpu' is DREAM's own CPU backend; this package implements "
            "device='cuda' only")
    raise RuntimeError("Error in das - unkown compute device string!")


def _report(status: int, name: str = "DAS") -> None:
    """Status -> the reference binding's behaviour (python/include/py_das.hpp:225-244)."""
    if status == _lib.STATUS_OOB:
        raise RuntimeError(f"{name} out-of-bounds!")
    if status == _lib.STATUS_WARN_OOB:
        print(f"Warning: {name} out-of-bounds!")


def _plan(key, create):
    cache = getattr(_tls, "plans", None)
    if cache is None:
        cache = _tls.plans = {}
    p = cache.get(key[0])
    if p is None or getattr(p, "cache_key", None) != key:
        cache.pop(key[0], None)
        p = create()
        p.cache_key = key  # the plan is reused while calls bring the same key
        cache[key[0]] = p
    return p


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _fortran(a, dtype) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=dtype))


def _rows_cols(a):
    s = tuple(a.shape)
    if len(s) == 0:
        return 1, 1
    if len(s) == 1:
        return s[0], 1
    if len(s) == 2:
        return s[0], s[1]
    raise RuntimeError("arguments must be vectors or matrices")


def _check_shapes(Y, Gt, Gr, Ro, delay, das_type, count_columns=True):
    """Shape checks of python/include/py_das.hpp:53-124, plus the A-scan count
    (the reference reads past Y when it has too few columns; here it is an error;
    count_columns=False leaves the count to the caller)."""
    K, C = _rows_cols(Y)
    if _rows_cols(Gt)[1] != 3:
        raise RuntimeError("Argument 2 must be a (num transmit elements) x 3 matrix!")
    Nt = _rows_cols(Gt)[0]
    Nr = 0
    if das_type != _lib.SAFT:
        if Gr is None or _rows_cols(Gr)[1] != 3:
            raise RuntimeError("Argument 3 must be a (num recieve elements) x 3 matrix!")
        Nr = _rows_cols(Gr)[0]
    if _rows_cols(Ro)[1] != 3:
        raise RuntimeError("Obs point error in das!")
    No = _rows_cols(Ro)[0]
    m, n = _rows_cols(delay)
    dlen = m * n
    if dlen < 1 or (dlen > 1 and dlen != No) or (dlen > 1 and not (m == 1 or n == 1)):
        raise RuntimeError("Error in das!")
    eff = _lib.SAFT if (das_type == _lib.SAFT or Nr == 0) else das_type
    need = Nt if eff == _lib.SAFT else Nt * Nr
    if count_columns and C < need:
        raise RuntimeError(f"das: Y has {C} A-scans but the method needs {need}")
    return K, No, Nt, Nr, (dlen > 1)


def das_generic(dtype, Y, Gt, Gr, Ro, dt, delay, cp, method, err_level="stop", device="cuda",
                verbose=""):
    """Shared body of ``das.das`` (FP64) and ``das_f.das`` (FP32)."""
    das_type = parse_method(method)
    level = parse_err_level(err_level)
    dev = parse_device(device)
    if _is_torch(Y):
        return _das_torch(dtype, Y, Gt, Gr, Ro, dt, delay, cp, das_type, level, dev)
    Y = _fortran(Y, dtype)
    Gt = _fortran(Gt, dtype)
    Gr = _fortran(Gr, dtype) if Gr is not None else None
    Ro = _fortran(Ro, dtype)
    delay = _fortran(delay, dtype)
    K, No, Nt, Nr, multi = _check_shapes(Y, Gt, Gr, Ro, delay, das_type)
    prec = _lib.PREC_F64 if np.dtype(dtype) == np.float64 else _lib.PREC_F32
    key = ("das", das_type, K, No, Nt, Nr, prec, dev)
    plan = _plan(key, lambda: _lib.plan_create(das_type, K, No, Nt, Nr, prec, dev))
    _set_hint(plan, grid_hint(Ro))
    Im = np.zeros(No, dtype=dtype)
    oob = ctypes.c_int64(0)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p) if a is not None and a.size else None
    st = _lib.check(_lib.load().dream_das_run(
        plan.handle, p(Y), p(Ro), p(Gt), p(Gr) if Nr else None, float(dt),
        _lib.DELAY_MULTIPLE if multi else _lib.DELAY_SINGLE, p(delay), float(cp),
        p(Im), level, ctypes.byref(oob)))
    _report(st)
    return Im


def _set_hint(plan, h):
    """The plan's grid hint (only speed depends on it: the plain kernels give
    each warp an 8 x 4 patch of the grid instead of 32 consecutive points)."""
    if getattr(plan, "hint", None) != h:
        _lib.check(_lib.load().dream_das_set_grid_hint(plan.handle, int(h)))
        plan.hint = h


def _torch_fortran(t, dtype, device):
    """Column-major device copy. Host data in pinned memory is uploaded
    asynchronously (the caller's stream orders it before the kernel)."""
    import torch
    tdt = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
    if not _is_torch(t):
        t = torch.as_tensor(np.asarray(t))
    if t.device.type == "cpu" and t.dtype == tdt:
        t = t.to(device=device, non_blocking=t.is_pinned())
    t = t.to(device=device, dtype=tdt)
    if t.dim() == 0:
        t = t.reshape(1, 1)
    if t.dim() == 1:
        t = t.reshape(-1, 1)
    # column-major storage: the transpose is row-major contiguous
    return t.t().contiguous().t()


def _das_torch(dtype, Y, Gt, Gr, Ro, dt, delay, cp, das_type, level, dev):
    import torch
    device = torch.device("cuda", dev) if Y.device.type != "cuda" else Y.device
    dev = device.index if device.index is not None else torch.cuda.current_device()
    Y = _torch_fortran(Y, dtype, device)
    Gt = _torch_fortran(Gt, dtype, device)
    Gr = _torch_fortran(Gr, dtype, device) if Gr is not None and das_type != _lib.SAFT else None
    Ro = _torch_fortran(Ro, dtype, device)
    delay = _torch_fortran(delay, dtype, device)
    K, No, Nt, Nr, multi = _check_shapes(Y, Gt, Gr, Ro, delay, das_type)
    prec = _lib.PREC_F64 if np.dtype(dtype) == np.float64 else _lib.PREC_F32
    key = ("das", das_type, K, No, Nt, Nr, prec, dev)
    plan = _plan(key, lambda: _lib.plan_create(das_type, K, No, Nt, Nr, prec, dev))
    _set_hint(plan, grid_hint(Ro))
    Im = torch.empty(No, dtype=Y.dtype, device=device)
    oob = ctypes.c_int64(0)
    stream = torch.cuda.current_stream(device).cuda_stream
    ptr = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() else None
    st = _lib.check(_lib.load().dream_das_run_device(
        plan.handle, ptr(Y), ptr(Ro), ptr(Gt), ptr(Gr), float(dt),
        _lib.DELAY_MULTIPLE if multi else _lib.DELAY_SINGLE, ptr(delay), float(cp), ptr(Im),
        level, ctypes.byref(oob), ctypes.c_void_p(stream)))
    _report(st)
    return Im


def das_uni(Y, gt, gr, ro, dt, delay, cp, method, err_level="ignore", device="cuda"):
    """``Im = das_uni(Y, gt, gr, ro, dt, delay, cp, method)`` on uniform grids.

    gt, gr: ``[min, pitch, max]`` (gr may be empty for SAFT); ro: 3x3 with rows
    x, y, z and columns (min, d, max). Precision follows Y (float32 -> FP32,
    otherwise FP64), like the Octave binding. Only the first delay value is
    used (opencl/cl_das_uni.cc is called with delay[0]).
    """
    das_type = parse_method(method)
    level = parse_err_level(err_level)
    dev = parse_device(device)
    is_t = _is_torch(Y)
    dtype = np.float32 if (str(Y.dtype).endswith("float32")) else np.float64
    gt = np.asarray(gt, dtype=np.float64).reshape(-1)
    gr = np.asarray(gr if gr is not None else [], dtype=np.float64).reshape(-1)
    ro = np.asarray(ro, dtype=np.float64)
    if gt.size != 3:
        raise RuntimeError("Argument 2 must be a 3 element vector")
    if gr.size not in (0, 3):
        raise RuntimeError("Argument 3 must be a 3 element vector!")
    if ro.shape != (3, 3):
        raise RuntimeError("Argument 4 must be a 3 x 3 matrix!")
    if gr.size == 0:
        if das_type != _lib.SAFT:
            raise RuntimeError("Argument 3 must be a 3 element vector!")
        gr = np.zeros(3)
    if dtype == np.float32:  # triplets in the kernel precision
        gt, gr, ro = (a.astype(np.float32).astype(np.float64) for a in (gt, gr, ro))
    tri = np.concatenate([gt, gr, ro[0], ro[1], ro[2]])
    d0 = float(np.asarray(delay.cpu() if _is_torch(delay) else delay, dtype=np.float64).reshape(-1)[0])
    prec = _lib.PREC_F64 if dtype == np.float64 else _lib.PREC_F32
    K = int(Y.shape[0])
    key = ("uni", das_type, K, tuple(tri.tolist()), prec, dev)
    plan = _plan(key, lambda: _lib.uni_plan_create(das_type, K, tri, prec, dev))
    L = _lib.load()
    No = L.dream_das_plan_num_points(plan.handle)
    need = L.dream_das_plan_num_ascans(plan.handle)
    if (int(Y.shape[1]) if len(Y.shape) > 1 else 1) < need:
        raise RuntimeError(f"das_uni: Y has too few A-scans (the grids need {need})")
    tri_c = (ctypes.c_double * 15)(*tri.tolist())
    oob = ctypes.c_int64(0)
    if is_t:
        import torch
        Yt = _torch_fortran(Y, dtype, Y.device if Y.device.type == "cuda" else torch.device("cuda", dev))
        Im = torch.empty(No, dtype=Yt.dtype, device=Yt.device)
        stream = torch.cuda.current_stream(Yt.device).cuda_stream
        st = _lib.check(L.dream_das_uni_run_device(plan.handle, ctypes.c_void_p(Yt.data_ptr()), tri_c,
                                                   float(dt), d0, float(cp), ctypes.c_void_p(Im.data_ptr()),
                                                   level, ctypes.byref(oob), ctypes.c_void_p(stream)))
    else:
        Yn = _fortran(Y, dtype)
        Im = np.zeros(No, dtype=dtype)
        st = _lib.check(L.dream_das_uni_run(plan.handle, Yn.ctypes.data_as(ctypes.c_void_p), tri_c, float(dt),
                                            d0, float(cp), Im.ctypes.data_as(ctypes.c_void_p), level,
                                            ctypes.byref(oob)))
    _report(st, "DAS_UNI")
    return Im


# ---------------------------------------------------------------------------
# Precision upgrade: FP32/BF16-stored A-scans, FP32 compensated sums, FP64-exact
# sample indices. Not part of the reference surface; same arguments plus
# `storage` and optional per-A-scan weights.
# ---------------------------------------------------------------------------

_STORAGE = {"f32": _lib.PREC_F32_STORE, "bf16": _lib.PREC_BF16_STORE}


def grid_hint(Ro) -> int:
    """Number of leading image points that share x and y (the fastest grid
    axis, e.g. Nz for ``meshgrid(x, z)`` flattened column-major), or 0 when
    it does not divide the number of points. Only speed depends on it, so
    the scan stops at the first change (growing windows of points)."""
    No = int(Ro.shape[0])
    if No == 0:
        return 0
    n, lo, win = No, 1, 1024
    while lo < No:
        hi = min(No, lo + win)
        blk = Ro[lo:hi]
        if _is_torch(Ro):
            import torch
            ch = torch.nonzero((blk[:, 0] != Ro[0, 0]) | (blk[:, 1] != Ro[0, 1]))
            if ch.numel():
                n = lo + int(ch[0, 0].item())
                break
        else:
            R = np.asarray(blk)
            ch = np.nonzero((R[:, 0] != Ro[0, 0]) | (R[:, 1] != Ro[0, 1]))[0]
            if ch.size:
                n = lo + int(ch[0])
                break
        lo, win = hi, win * 4
    return n if (n > 0 and No % n == 0 and n < No) else 0


def _fast_plan(das_type, K, No, Nt, Nr, prec, dev, hint, tile=None):
    key = ("fast", das_type, K, No, Nt, Nr, prec, dev)
    plan = _plan(key, lambda: _lib.plan_create(das_type, K, No, Nt, Nr, prec, dev))
    L = _lib.load()
    if getattr(plan, "hint", None) != hint:
        _lib.check(L.dream_das_set_grid_hint(plan.handle, int(hint)))
        plan.hint = hint
        plan.tile = None
    if tile is not None and getattr(plan, "tile", None) != tuple(tile):
        _lib.check(L.dream_das_set_tile(plan.handle, int(tile[0]), int(tile[1])))
        plan.tile = tuple(tile)
    return plan


def _das_mixed_host(Y, Gt, Gr, Ro, dt, delay, cp, das_type, level, dev, prec, hint, tile):
    """Host arrays through the C ABI's host entry (dream_das_run): FP32
    A-scans, FP64 geometry, column-major. For TFM and RCA frames of 8 MB or
    more the library uploads the A-scans in chunks of inner elements on a copy
    stream and beamforms each chunk as it lands, so the upload (the larger part
    of an end-to-end call) overlaps the kernels; pinned host memory makes the
    copies run at full link speed."""
    host = lambda a: a.numpy() if _is_torch(a) else a
    Yh = _fortran(host(Y), np.float32)
    Gth = _fortran(host(Gt), np.float64)
    Grh = _fortran(host(Gr), np.float64) if Gr is not None and das_type != _lib.SAFT else None
    Roh = _fortran(host(Ro), np.float64)
    dlh = _fortran(host(delay), np.float64)
    if Yh.ndim == 1:
        Yh = Yh.reshape(-1, 1, order="F")
    K, No, Nt, Nr, multi = _check_shapes(Yh, Gth, Grh, Roh, dlh, das_type)
    h = grid_hint(Roh) if hint == "auto" else int(hint or 0)
    plan = _fast_plan(das_type, K, No, Nt, Nr, prec, dev, h, tile)
    # the image lands in page-locked memory from torch's caching host
    # allocator (the array keeps its block alive): the read-back runs at link
    # speed without a staging copy
    import torch
    out = torch.empty(No, dtype=torch.float32, pin_memory=True).numpy()
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p) if a is not None and a.size else None
    oob = ctypes.c_int64(0)
    st = _lib.check(_lib.load().dream_das_run(
        plan.handle, ptr(Yh), ptr(Roh), ptr(Gth), ptr(Grh), float(dt),
        _lib.DELAY_MULTIPLE if multi else _lib.DELAY_SINGLE, ptr(dlh), float(cp), ptr(out), level,
        ctypes.byref(oob)))
    _report(st)
    return out


def inner_count(das_type: int, Nt: int, Nr: int) -> tuple:
    """(outer, inner) element counts of a TFM / RCA frame: RCA row-tx loops
    over rows (Gr) outside and columns (Gt) inside, the others Gt outside."""
    return (Nr, Nt) if das_type == _lib.RCA_ROWTX else (Nt, Nr)


def das_mixed(Y, Gt, Gr, Ro, dt, delay, cp, method, err_level="stop", device="cuda", storage="f32",
              weights=None, hint="auto", tile=None, stream=None, inner=None):
    """DAS with A-scans stored in FP32 (``storage='f32'``) or BF16 and FP32
    compensated accumulation; sample indices are the FP64 reference's.

    Geometry and delays are taken in FP64. Returns an FP32 image (a torch
    tensor on the device when Y is a CUDA tensor, else a NumPy array).
    ``weights`` (one per A-scan column) gives ``sum_c w[c] * Y[k, c]``.
    ``inner=(lo, hi)``: Y holds only the A-scans of inner elements [lo, hi)
    (column o * (hi - lo) + i - lo; see ``inner_count``) and the result is the
    partial image over those terms (dream_das_set_inner_shard).
    """
    import torch
    das_type = parse_method(method)
    level = parse_err_level(err_level)
    dev = parse_device(device)
    prec = _STORAGE[storage]
    on_host = not (_is_torch(Y) and Y.device.type == "cuda")
    if on_host and weights is None and stream is None and inner is None:
        return _das_mixed_host(Y, Gt, Gr, Ro, dt, delay, cp, das_type, level, dev, prec, hint, tile)
    device_t = Y.device if not on_host else torch.device("cuda", dev)
    dev = device_t.index if device_t.index is not None else torch.cuda.current_device()
    ydt = np.float32
    Yt = _torch_fortran(Y, ydt, device_t)
    if prec == _lib.PREC_BF16_STORE:
        Yt = Yt.t().contiguous().to(torch.bfloat16).t()
    Gt_t = _torch_fortran(Gt, np.float64, device_t)
    Gr_t = _torch_fortran(Gr, np.float64, device_t) if Gr is not None and das_type != _lib.SAFT else None
    Ro_t = _torch_fortran(Ro, np.float64, device_t)
    dl_t = _torch_fortran(delay, np.float64, device_t)
    if inner is not None and weights is not None:
        raise RuntimeError("das: weights and an inner-element shard cannot be combined")
    if inner is None:
        K, No, Nt, Nr, multi = _check_shapes(Yt, Gt_t, Gr_t, Ro_t, dl_t, das_type)
    else:
        lo, hi = int(inner[0]), int(inner[1])
        K, C = _rows_cols(Yt)
        _, No, Nt, Nr, multi = _check_shapes(Yt, Gt_t, Gr_t, Ro_t, dl_t, das_type, count_columns=False)
        n_out, n_in = inner_count(das_type, Nt, Nr)
        if das_type == _lib.SAFT or not (0 <= lo < hi <= n_in):
            raise RuntimeError("das: inner-element shard out of range")
        if C != n_out * (hi - lo):
            raise RuntimeError(f"das: an inner-element shard [{lo}, {hi}) needs {n_out * (hi - lo)} A-scans, got {C}")
    h = grid_hint(Ro if not on_host else np.asarray(Ro)) if hint == "auto" else int(hint or 0)
    plan = _fast_plan(das_type, K, No, Nt, Nr, prec, dev, h, tile)
    Im = torch.empty(No, dtype=torch.float32, device=device_t)
    d_oob = torch.zeros(1, dtype=torch.int64, device=device_t)
    st_ = stream if stream is not None else torch.cuda.current_stream(device_t).cuda_stream
    ptr = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() else None
    L = _lib.load()
    common = (plan.handle, ptr(Yt), ptr(Ro_t), ptr(Gt_t), ptr(Gr_t), float(dt),
              _lib.DELAY_MULTIPLE if multi else _lib.DELAY_SINGLE, ptr(dl_t), float(cp))
    if weights is not None:
        w = torch.as_tensor(weights, dtype=torch.float32, device=device_t).reshape(-1).contiguous()
        need = Nt if (das_type == _lib.SAFT or Nr == 0) else Nt * Nr
        if w.numel() != need:
            raise RuntimeError(f"das: weights need {need} values (one per A-scan column)")
        _lib.check(L.dream_das_weighted_run_device(*common, ptr(w), ptr(Im), ptr(d_oob),
                                                   ctypes.c_void_p(st_)))
    elif inner is not None:
        _lib.check(L.dream_das_set_inner_shard(plan.handle, lo, hi))
        try:
            _lib.check(L.dream_das_run_device_async(*common, ptr(Im), ptr(d_oob), ctypes.c_void_p(st_)))
        finally:
            _lib.check(L.dream_das_set_inner_shard(plan.handle, 0, 0))
    else:
        _lib.check(L.dream_das_run_device_async(*common, ptr(Im), ptr(d_oob), ctypes.c_void_p(st_)))
    oob = int(d_oob.item())
    st = 0 if oob == 0 else {_lib.LVL_IGNORE: 1, _lib.LVL_WARN: 2, _lib.LVL_STOP: 3}[level]
    _report(st)
    return Im.cpu().numpy() if on_host else Im
