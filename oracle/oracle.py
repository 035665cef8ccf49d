"""ctypes front end of the C restatement of the reference DAS (das_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker. The product path never imports it.

Also exposes the unmodified reference modules built by oracle/build_ref.sh
(``reference_module``) when they are present.
"""
from __future__ import annotations

import ctypes
import glob
import importlib.util
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdas_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

METHODS = {"saft": 0, "tfm": 1, "rca": 2, "rca_coltx": 2, "rca_rowtx": 3}
ERR_LEVELS = {"none": 0, "ignore": 1, "warn": 2, "stop": 3}
OOB_MISS = np.iinfo(np.int64).min

_lib = None


def build() -> str:
    """Compiles das_oracle.c and conv_oracle.c with gcc (make) if the shared object is stale."""
    srcs = [os.path.join(HERE, f) for f in ("das_oracle.c", "conv_oracle.c", "rect_oracle.c")]
    if (not os.path.exists(LIB_PATH)) or os.path.getmtime(LIB_PATH) < max(os.path.getmtime(f) for f in srcs):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        i64, i32, vp = ctypes.c_int64, ctypes.c_int, ctypes.c_void_p
        f64, f32 = ctypes.c_double, ctypes.c_float
        L.dream_oracle_das_f64.argtypes = [i32, vp, i64, vp, i64, vp, i64, vp, i64, f64, i32, vp,
                                           f64, i32, vp, vp, vp]
        L.dream_oracle_das_f32.argtypes = [i32, vp, i64, vp, i64, vp, i64, vp, i64, f32, i32, vp,
                                           f32, i32, vp, vp, vp]
        L.dream_oracle_das_uni_f64.argtypes = [i32, vp, i64, vp, f64, f64, f64, i32, vp, vp]
        L.dream_oracle_das_uni_f32.argtypes = [i32, vp, i64, vp, f32, f32, f32, i32, vp, vp]
        L.dream_oracle_uni_count_f64.argtypes = [f64, f64, f64]
        L.dream_oracle_uni_count_f64.restype = i64
        L.dream_oracle_uni_count_f32.argtypes = [f32, f32, f32]
        L.dream_oracle_uni_count_f32.restype = i64
        for n in ("dream_oracle_das_weighted_f64", "dream_oracle_das_adjoint_f64"):
            getattr(L, n).argtypes = [vp, i64, i64, i64, vp, vp, vp]
        L.dream_oracle_das_wgrad_f64.argtypes = [vp, i64, i64, i64, vp, vp, vp]
        L.dream_oracle_conv_p.argtypes = [vp, i64, i64, vp, i64, i64, vp, i32]
        L.dream_oracle_conv_p.restype = None
        L.dream_oracle_rect.argtypes = [vp, i64, f64, f64, f64, f64, f64, i64, i32, vp, f64, f64, i32, vp, vp]
        L.dream_oracle_rect.restype = i32
        L.dream_oracle_arr_elements.argtypes = [vp, i64, i32, vp, i32, f64, f64, i32, vp, f64, f64, vp, vp, vp]
        L.dream_oracle_arr_elements.restype = None
        L.dream_oracle_arr_rect.argtypes = [vp, i64, f64, f64, f64, f64, f64, i64, i32, vp, f64, f64, i64, vp, i32,
                                            vp, i32, f64, f64, i32, vp, f64, i32, vp, vp]
        L.dream_oracle_arr_rect.restype = i32
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def das(Y, Gt, Gr, Ro, dt, delay, cp, method="tfm", err_level="ignore", dtype=np.float64,
        return_idx=False):
    """Oracle ``das``: returns ``(Im, status, oob_count[, idx])``.

    ``dtype`` float64 restates ``das`` (DAS<double>), float32 restates
    ``das_f`` (DAS<float>). ``idx`` is ``(terms, No)`` int64 with
    ``OOB_MISS`` for out-of-bounds terms.
    """
    dt_ = np.dtype(dtype)
    c = lambda a: np.asfortranarray(np.asarray(a, dtype=dt_))
    Y, Gt, Ro = c(Y), c(Gt), c(Ro)
    Gr = c(Gr) if Gr is not None and np.size(Gr) else np.zeros((0, 3), dtype=dt_, order="F")
    delay = c(np.atleast_1d(np.asarray(delay)).reshape(-1))
    K, No, Nt = Y.shape[0], Ro.shape[0], Gt.shape[0]
    m = METHODS[method]
    Nr = 0 if m == 0 else Gr.shape[0]
    if Nr == 0:
        m = 0
    multi = 1 if delay.size != 1 else 0
    Im = np.zeros(No, dtype=dt_)
    oob = ctypes.c_int64(0)
    idx = None
    if return_idx:
        terms = Nt if m == 0 else Nt * Nr
        idx = np.zeros((terms, No), dtype=np.int64)
    fn = lib().dream_oracle_das_f64 if dt_ == np.float64 else lib().dream_oracle_das_f32
    st = fn(m, _p(Y), K, _p(Ro), No, _p(Gt), Nt, _p(Gr), Nr, dt, multi, _p(delay), cp,
            ERR_LEVELS[err_level], _p(Im), ctypes.byref(oob), _p(idx))
    if return_idx:
        return Im, st, oob.value, idx
    return Im, st, oob.value


def uni_count(mn, d, mx, dtype=np.float64) -> int:
    if np.dtype(dtype) == np.float64:
        return int(lib().dream_oracle_uni_count_f64(mn, d, mx))
    return int(lib().dream_oracle_uni_count_f32(mn, d, mx))


def das_uni(Y, gt, gr, ro, dt, delay, cp, method="tfm", err_level="ignore", dtype=np.float64):
    """Oracle ``das_uni`` (the reference's OpenCL kernels restated on the CPU).

    ``gt``/``gr`` are ``[min, pitch, max]``; ``ro`` is 3x3 with rows x, y, z and
    columns (min, d, max). Returns ``(Im, status, oob_count)``.
    """
    dt_ = np.dtype(dtype)
    Y = np.asfortranarray(np.asarray(Y, dtype=dt_))
    gt = np.asarray(gt, dtype=dt_).reshape(-1)
    gr = np.asarray(gr, dtype=dt_).reshape(-1) if gr is not None and np.size(gr) else np.zeros(3, dt_)
    ro = np.asarray(ro, dtype=dt_).reshape(3, 3)
    tri = np.concatenate([gt, gr, ro[0], ro[1], ro[2]]).astype(dt_)
    m = METHODS[method]
    if m != 0 and np.size(gr) == 0:
        m = 0
    cnt = lambda a, b, c: uni_count(a, b, c, dt_)
    No = cnt(*ro[0]) * cnt(*ro[1]) * cnt(*ro[2])
    Im = np.zeros(No, dtype=dt_)
    oob = ctypes.c_int64(0)
    fn = lib().dream_oracle_das_uni_f64 if dt_ == np.float64 else lib().dream_oracle_das_uni_f32
    d0 = float(np.asarray(delay).reshape(-1)[0])
    st = fn(m, _p(Y), Y.shape[0], _p(tri), dt, d0, cp, ERR_LEVELS[err_level], _p(Im),
            ctypes.byref(oob))
    return Im, st, oob.value


def weighted(idx, Y, w):
    """``Im[o] = sum_c w[c] * Y[idx[c, o], c]`` on an oracle index table."""
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    Y = np.asfortranarray(Y, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64).reshape(-1)
    C, No = idx.shape
    Im = np.zeros(No)
    lib().dream_oracle_das_weighted_f64(_p(idx), No, C, Y.shape[0], _p(Y), _p(w), _p(Im))
    return Im


def adjoint(idx, x, w, K):
    """``Ya[idx[c, o], c] += w[c] * x[o]``: the adjoint of :func:`weighted`."""
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    w = np.ascontiguousarray(w, dtype=np.float64).reshape(-1)
    C, No = idx.shape
    Ya = np.zeros((K, C), order="F")
    lib().dream_oracle_das_adjoint_f64(_p(idx), No, C, K, _p(x), _p(w), _p(Ya))
    return Ya


def wgrad(idx, g, Y):
    """``dw[c] = sum_o g[o] * Y[idx[c, o], c]``."""
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    g = np.ascontiguousarray(g, dtype=np.float64).reshape(-1)
    Y = np.asfortranarray(Y, dtype=np.float64)
    C, No = idx.shape
    dw = np.zeros(C)
    lib().dream_oracle_das_wgrad_f64(_p(idx), No, C, Y.shape[0], _p(g), _p(Y), _p(dw))
    return dw


def reference_module(precision: str = "f64"):
    """The unmodified reference module (``das`` or ``das_f``) from oracle/_ref, or None."""
    name = "das" if precision == "f64" else "das_f"
    hits = glob.glob(os.path.join(REF_DIR, name + ".cpython-*.so"))
    if not hits:
        return None
    spec = importlib.util.spec_from_file_location(name, hits[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


CONV_MODES = {"=": 0, "+=": 1, "-=": 2}


def conv_p(A, B, Y=None, mode="="):
    """Column-wise full linear convolution, the direct form of the reference's
    conv() (conv_oracle.c; pinned against the reference's own conv(), see
    reference_conv_p).
    Returns Y ((A_M + B_M - 1) x A_N, FP64, column-major); with Y given it is
    updated in place by mode '=', '+=' or '-='."""
    A = np.asfortranarray(np.asarray(A, dtype=np.float64))
    B = np.asfortranarray(np.asarray(B, dtype=np.float64))
    if A.ndim == 1:
        A = A.reshape(-1, 1, order="F")
    A_M, A_N = A.shape
    B_M, B_N = (B.shape[0], B.shape[1]) if B.ndim == 2 else (B.shape[0], 1)
    if B_M == 1 or B_N == 1:
        B_M, B_N = B_M * B_N, 1
    elif B_N != A_N:
        raise RuntimeError("Argument 2 must be a vector or a matrix with the same number of columns as arg 1!")
    if Y is None:
        Y = np.zeros((A_M + B_M - 1, A_N), dtype=np.float64, order="F")
    assert Y.flags["F_CONTIGUOUS"] and Y.dtype == np.float64 and Y.shape == (A_M + B_M - 1, A_N)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    lib().dream_oracle_conv_p(p(A), A_M, A_N, p(B), B_M, B_N, p(Y), CONV_MODES[mode])
    return Y


def rect(Ro, a, b, dx, dy, dt, nt, delay, v, cp, err_level="ignore"):
    """Oracle dreamrect (rect_oracle.c, no attenuation): returns
    ``(H, status, oob)``, H nt x No FP64 column-major."""
    Ro = np.asfortranarray(np.asarray(Ro, dtype=np.float64))
    delay = np.ascontiguousarray(np.asarray(delay, dtype=np.float64).reshape(-1))
    No = Ro.shape[0]
    H = np.zeros((int(nt), No), dtype=np.float64, order="F")
    oob = ctypes.c_int64(0)
    st = lib().dream_oracle_rect(_p(Ro), No, a, b, dx, dy, dt, int(nt), int(delay.size > 1), _p(delay), v, cp,
                                 ERR_LEVELS[err_level], _p(H), ctypes.byref(oob))
    return H, st, oob.value


def reference_rect(Ro, a, b, dx, dy, dt, nt, delay, v, cp):
    """The reference's OpenCL dreamrect kernel compiled as C (oracle/_ref,
    built by build_ref.sh from the reference sources), or None when absent."""
    path = os.path.join(REF_DIR, "libref_dreamrect.so")
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    L.dream_ref_dreamrect.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_double] * 5 + \
        [ctypes.c_int] + [ctypes.c_double] * 3 + [ctypes.c_void_p]
    Ro = np.asfortranarray(np.asarray(Ro, dtype=np.float64))
    H = np.zeros((int(nt), Ro.shape[0]), dtype=np.float64, order="F")
    L.dream_ref_dreamrect(_p(Ro), Ro.shape[0], a, b, dx, dy, dt, int(nt), float(delay), v, cp, _p(H))
    return H


# Method codes of the array entries (include/dream_sir.h), by the reference's strings.
FOC_METHODS = {"off": 0, "x": 1, "y": 2, "xy": 3, "on": 3, "x+y": 4, "ud": 5}
STEER_METHODS = {"off": 0, "x": 1, "y": 2, "xy": 3}
APOD_METHODS = {"off": 0, "triangle": 1, "gauss": 2, "raised": 3, "hann": 4, "hamming": 5, "simply": 6,
                "clamped": 7, "ud": 8}


def _arr_args(G, focal, apod):
    G = np.asfortranarray(np.asarray(G, dtype=np.float64))
    focal = np.ascontiguousarray(np.asarray(focal, dtype=np.float64).reshape(-1))
    apod = None if apod is None else np.ascontiguousarray(np.asarray(apod, dtype=np.float64).reshape(-1))
    return G, focal, apod


def arr_elements(G, foc_met, focal, steer_met, theta, phi, apod_met, apod, apod_par, cp, reference=False):
    """Per-element focusing delays, steering delays and weights of an array:
    ``(foc, steer, weight)``. ``reference=True`` runs the reference's own
    src/arr_functions.cc (oracle/_ref/libref_arr.so; None when absent)
    instead of the restatement in rect_oracle.c."""
    G, focal, apod = _arr_args(G, focal, apod)
    M = G.shape[0]
    out = [np.zeros(M) for _ in range(3)]
    args = (_p(G), M, FOC_METHODS[foc_met], _p(focal), STEER_METHODS[steer_met], float(theta), float(phi),
            APOD_METHODS[apod_met], _p(apod), float(apod_par), float(cp), *[_p(o) for o in out])
    if reference:
        path = os.path.join(REF_DIR, "libref_arr.so")
        if not os.path.exists(path):
            return None
        L = ctypes.CDLL(path)
        L.dream_ref_arr_elements.argtypes = lib().dream_oracle_arr_elements.argtypes
        L.dream_ref_arr_elements.restype = None
        L.dream_ref_arr_elements(*args)
    else:
        lib().dream_oracle_arr_elements(*args)
    return tuple(out)


def arr_rect(Ro, a, b, G, dx, dy, dt, nt, delay, v, cp, foc_met="off", focal=0.0, steer_met="off", theta=0.0,
             phi=0.0, apod_met="off", apod=None, apod_par=0.0, err_level="ignore"):
    """Oracle dream_arr_rect (rect_oracle.c, no attenuation): returns
    ``(H, status, oob)``, H nt x No FP64 column-major."""
    Ro = np.asfortranarray(np.asarray(Ro, dtype=np.float64))
    G, focal, apod = _arr_args(G, focal, apod)
    delay = np.ascontiguousarray(np.asarray(delay, dtype=np.float64).reshape(-1))
    No = Ro.shape[0]
    H = np.zeros((int(nt), No), dtype=np.float64, order="F")
    oob = ctypes.c_int64(0)
    st = lib().dream_oracle_arr_rect(_p(Ro), No, a, b, dx, dy, dt, int(nt), int(delay.size > 1), _p(delay), v, cp,
                                     G.shape[0], _p(G), FOC_METHODS[foc_met], _p(focal), STEER_METHODS[steer_met],
                                     float(theta), float(phi), APOD_METHODS[apod_met], _p(apod), float(apod_par),
                                     ERR_LEVELS[err_level], _p(H), ctypes.byref(oob))
    return H, st, oob.value

# ---------------------------------------------------------------------------
# The reference's own CPU code (oracle/_ref/libref_cpu.so, built unmodified by
# build_ref.sh with FFTW replaced by oracle/fftw_stub.c): conv() of
# extra_src/conv.cc, Rect::dreamrect of src/dreamrect.cc and
# ArrRect::dream_arr_rect of src/dream_arr_rect.cc, without attenuation.
# Each returns None when the library is absent.
# ---------------------------------------------------------------------------

_ref_cpu = None


def reference_cpu():
    global _ref_cpu
    if _ref_cpu is None:
        path = os.path.join(REF_DIR, "libref_cpu.so")
        if not os.path.exists(path):
            return None
        L = ctypes.CDLL(path)
        vp, i64, f64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int
        L.dream_ref_conv.argtypes = [vp, i64, vp, i64, vp, i32]
        L.dream_ref_conv.restype = None
        L.dream_ref_dreamrect.argtypes = [vp, i64, f64, f64, f64, f64, f64, i64, i32, vp, f64, f64, i32, vp]
        L.dream_ref_dreamrect.restype = i32
        L.dream_ref_arr_rect.argtypes = [vp, i64, f64, f64, f64, f64, f64, i64, i32, vp, f64, f64, i64, vp, i32, vp,
                                         i32, f64, f64, i32, vp, f64, i32, vp]
        L.dream_ref_arr_rect.restype = i32
        _ref_cpu = L
    return _ref_cpu


CONV_MODES = {"=": 0, "+=": 1, "-=": 2}


def reference_conv_p(A, B, Y=None, mode="="):
    """Column-wise conv() of the reference (extra_src/conv.cc:33-78) as
    conv_p calls it: column n of A convolved with column n of B (or with the
    single column B); ``Y`` is updated in place for '+=' / '-='."""
    L = reference_cpu()
    if L is None:
        return None
    A = np.asfortranarray(np.asarray(A, dtype=np.float64))
    B = np.asfortranarray(np.asarray(B, dtype=np.float64))
    if A.ndim == 1:
        A = A.reshape(-1, 1, order="F")
    if B.ndim == 1:
        B = B.reshape(-1, 1, order="F")
    M, N = A.shape
    Lb, nb = B.shape
    if Y is None:
        Y = np.zeros((M + Lb - 1, N), order="F")
    else:
        Y = np.asfortranarray(np.array(Y, dtype=np.float64))
    for n in range(N):
        a = np.ascontiguousarray(A[:, n])
        b = np.ascontiguousarray(B[:, n if nb > 1 else 0])
        y = np.ascontiguousarray(Y[:, n])
        L.dream_ref_conv(_p(a), M, _p(b), Lb, _p(y), CONV_MODES[mode])
        Y[:, n] = y
    return Y


def reference_dreamrect(Ro, a, b, dx, dy, dt, nt, delay, v, cp, err_level="ignore"):
    """The reference's CPU dreamrect: ``(H, status)``, H nt x No."""
    L = reference_cpu()
    if L is None:
        return None
    Ro = np.asfortranarray(np.asarray(Ro, dtype=np.float64))
    delay = np.ascontiguousarray(np.asarray(delay, dtype=np.float64).reshape(-1))
    H = np.zeros((int(nt), Ro.shape[0]), dtype=np.float64, order="F")
    st = L.dream_ref_dreamrect(_p(Ro), Ro.shape[0], a, b, dx, dy, dt, int(nt), int(delay.size > 1), _p(delay), v, cp,
                               ERR_LEVELS[err_level], _p(H))
    return H, st


def reference_arr_rect(Ro, a, b, G, dx, dy, dt, nt, delay, v, cp, foc_met="off", focal=0.0, steer_met="off",
                       theta=0.0, phi=0.0, apod_met="off", apod=None, apod_par=0.0, err_level="ignore"):
    """The reference's CPU dream_arr_rect (arguments as arr_rect): ``(H, status)``."""
    L = reference_cpu()
    if L is None:
        return None
    Ro = np.asfortranarray(np.asarray(Ro, dtype=np.float64))
    G, focal, apod = _arr_args(G, focal, apod)
    if apod is None:
        apod = np.ones(G.shape[0])
    if focal.size < G.shape[0]:
        focal = np.resize(focal, G.shape[0])  # the reference reads focal[n] for 'ud' only
    delay = np.ascontiguousarray(np.asarray(delay, dtype=np.float64).reshape(-1))
    H = np.zeros((int(nt), Ro.shape[0]), dtype=np.float64, order="F")
    st = L.dream_ref_arr_rect(_p(Ro), Ro.shape[0], a, b, dx, dy, dt, int(nt), int(delay.size > 1), _p(delay), v, cp,
                              G.shape[0], _p(G), FOC_METHODS[foc_met], _p(focal), STEER_METHODS[steer_met],
                              float(theta), float(phi), APOD_METHODS[apod_met], _p(apod), float(apod_par),
                              ERR_LEVELS[err_level], _p(H))
    return H, st
