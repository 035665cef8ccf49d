"""``dreamrect`` and ``dream_arr_rect`` on the GPU: spatial impulse responses
of a rectangular transducer and of an array of rectangular elements, the
CUDA counterparts of the reference modules ``dreamrect``
(python/src/py_dreamrect.cc:47-139; src/dreamrect.cc, opencl/dreamrect.cl)
and ``dream_arr_rect`` (python/src/py_dream_arr_rect.cc:46-227;
src/dream_arr_rect.cc, src/arr_functions.cc).

    H = dreamrect(Ro, geom_par, s_par, delay, m_par, err_level="stop", device="cuda")
    H = dream_arr_rect(Ro, geom_par, G, s_par, delay, m_par, foc_met, focal, steer_met, steer_par,
                       apod_met, apod, win_par, err_level="stop", device="cuda")

Ro: No x 3 observation points (mm). geom_par = [a, b]: element size (mm).
s_par = [dx, dy, dt, nt]: surface discretisation (mm), sampling period (us),
SIR length. delay (us): a scalar or one value per point. m_par = [v, cp,
alpha]: normal velocity, sound speed (m/s), attenuation (only alpha = 0: the
reference's attenuation filter has no CUDA counterpart). Returns H, nt x No
FP64 column-major (a CUDA tensor when Ro is one), equal to the reference's
bit for bit. err_level 'ignore' / 'warn' / 'stop' treats samples outside
[0, nt) as the reference does ('stop' raises).

Arrays: G (num_elements x 3, mm) holds the element centres; foc_met "off",
"x", "y", "xy" (or "on"), "x+y" with focal the focal depth (mm, a scalar),
or "ud" with focal one delay (us) per element; steer_met "off", "x", "y",
"xy" with steer_par = [theta, phi] (degrees); apod_met "off", "triangle",
"gauss", "raised", "hann", "hamming", "simply", "clamped", or "ud" with apod
one weight per element. win_par is accepted and, as in the reference's
Python binding, not used: the shape parameter of "gauss" and "raised" is 0.
"""
from __future__ import annotations

import ctypes
import sys

import numpy as np

from . import _lib
from .beamformer import _is_torch, parse_device, parse_err_level

FOC_METHODS = {"off": 0, "x": 1, "y": 2, "xy": 3, "on": 3, "x+y": 4, "ud": 5}
STEER_METHODS = {"off": 0, "x": 1, "y": 2, "xy": 3}
APOD_METHODS = {"off": 0, "triangle": 1, "gauss": 2, "raised": 3, "hann": 4, "hamming": 5, "simply": 6,
                "clamped": 7, "ud": 8}


def _fail(fn, msg):
    sys.stderr.write(msg + "\n")
    raise RuntimeError(f"Error in {fn}!")


def _host(p):
    return np.asarray(p.cpu() if _is_torch(p) else p, dtype=np.float64)


def _vector(fn, p, n, what):
    a = _host(p)
    if not (a.size == n and (a.ndim <= 1 or (a.ndim == 2 and 1 in a.shape))):
        _fail(fn, f"{fn} requires that {what} must be a {n} element vector!")
    return a.reshape(-1)


def _common(fn, Ro, geom_par, s_par, delay, m_par, err_level):
    """Argument checks shared by dreamrect and dream_arr_rect, as the
    reference's ArgParser (include/arg_parser_python.h) makes them."""
    shape = tuple(Ro.shape)
    if len(shape) != 2 or shape[1] != 3:
        _fail(fn, f"{fn} requires that observation point arg must be a (number of observation points) x 3 matrix!")
    No = shape[0]
    a, b = _vector(fn, geom_par, 2, "the geometry arg")
    dx, dy, dt, nt_f = _vector(fn, s_par, 4, "sampling par arg")
    v, cp, alpha = _vector(fn, m_par, 3, "material parameters par arg")
    if alpha > np.finfo(np.float64).eps:
        raise RuntimeError(f"{fn}: attenuation (alpha > 0) is not supported by the CUDA backend")
    d = _host(delay)
    if d.size > 1 and (d.size != No or not (d.ndim <= 1 or 1 in d.shape)):
        _fail(fn, f"{fn} requires that delay arg must be a {d.size} element vector (with a length equal to "
                  "the number of observation points) or a scalar!")
    if d.size < 1:
        _fail(fn, f"{fn} requires a delay")
    return dict(No=No, a=a, b=b, dx=dx, dy=dy, dt=dt, nt=int(nt_f), v=v, cp=cp, d=d.reshape(-1),
                level=parse_err_level(err_level))


def _run(fn, Ro, c, device, arr=None):
    """One call of the C ABI (device entry for CUDA tensors, host entry for
    arrays); arr holds the array arguments (None: dreamrect)."""
    L = _lib.load()
    No, nt = c["No"], c["nt"]
    multi = _lib.DELAY_MULTIPLE if c["d"].size > 1 else _lib.DELAY_SINGLE
    geom = (c["a"], c["b"], c["dx"], c["dy"], c["dt"], nt, multi)
    oob = ctypes.c_int64(0)
    hp = lambda x: x.ctypes.data_as(ctypes.c_void_p) if x is not None and x.size else None
    arr_args = ()
    if arr is not None:
        arr_args = (arr["M"], hp(arr["G"]), arr["foc"], hp(arr["focal"]), arr["steer"], arr["theta"], arr["phi"],
                    arr["apod_met"], hp(arr["apod"]), arr["apod_par"])
    if _is_torch(Ro) and Ro.device.type == "cuda":
        import torch
        dev = Ro.device
        Rt = Ro.to(torch.float64).t().contiguous().t()
        dt_ = torch.as_tensor(c["d"], device=dev)
        H = torch.empty((No, nt), dtype=torch.float64, device=dev).t()
        p = lambda t: ctypes.c_void_p(t.data_ptr()) if t.numel() else None
        tail = (p(H), c["level"], ctypes.byref(oob), dev.index if dev.index is not None else 0,
                ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
        head = (p(Rt), No) + geom + (p(dt_), c["v"], c["cp"])
        st = (L.dream_arr_rect_run_device(*head, *arr_args, *tail) if arr is not None
              else L.dream_rect_run_device(*head, *tail))
    else:
        Rh = np.asfortranarray(np.asarray(Ro, dtype=np.float64))
        dh = np.ascontiguousarray(c["d"])
        H = np.zeros((nt, No), dtype=np.float64, order="F")
        head = (hp(Rh), No) + geom + (hp(dh), c["v"], c["cp"])
        tail = (hp(H), c["level"], ctypes.byref(oob), parse_device(device))
        st = L.dream_arr_rect_run(*head, *arr_args, *tail) if arr is not None else L.dream_rect_run(*head, *tail)
    _lib.check(st)
    if st == _lib.STATUS_OOB:
        _fail(fn, "SIR out-of-bounds!")
    if st == _lib.STATUS_WARN_OOB:
        print("Warning: SIR out-of-bounds!")
    return H


def dreamrect(Ro, geom_par, s_par, delay, m_par, err_level="stop", device="cuda"):
    c = _common("dreamrect", Ro, geom_par, s_par, delay, m_par, err_level)
    return _run("dreamrect", Ro, c, device)


def dream_arr_rect(Ro, geom_par, G, s_par, delay, m_par, foc_met, focal, steer_met, steer_par, apod_met, apod,
                   win_par, err_level="stop", device="cuda"):
    fn = "dream_arr_rect"
    c = _common(fn, Ro, geom_par, s_par, delay, m_par, err_level)
    Gh = _host(G)
    if Gh.ndim != 2 or Gh.shape[1] != 3:
        _fail(fn, f"{fn} requires that array grid arg must be a (number of array elements) x 3 matrix!")
    M = Gh.shape[0]
    if foc_met not in FOC_METHODS:
        _fail(fn, f"{fn} Unknown focusing method!")
    fh = _host(focal).reshape(-1)
    if foc_met == "ud":
        if fh.size != M:
            _fail(fn, f"{fn} the time delay vector arg for user defined ('ud') focusing\n!delays must have the "
                      "same length as the number of array elements!")
    elif fh.size != 1:
        _fail(fn, f"{fn} arg must be a scalar for non-user defined focusing!")
    if steer_met not in STEER_METHODS:
        _fail(fn, f"{fn} Unknown beem steering method!")
    sp = _host(steer_par)
    if not (sp.size == 2 and (sp.ndim <= 1 or (sp.ndim == 2 and 1 in sp.shape))):
        _fail(fn, f"{fn} steer_par must be a 2 element vector!")
    theta, phi = sp.reshape(-1)
    if apod_met not in APOD_METHODS:
        _fail(fn, f"{fn} Unknown apodization method!")
    ah = None
    if apod_met == "ud":
        ah = _host(apod).reshape(-1)
        if ah.size != M:
            _fail(fn, f"{fn} the length of apodization vector argument must be the same as the number of array "
                      "elements!")
        ah = np.ascontiguousarray(ah)
    arr = dict(M=M, G=np.asfortranarray(Gh), foc=FOC_METHODS[foc_met], focal=np.ascontiguousarray(fh),
               steer=STEER_METHODS[steer_met], theta=float(theta), phi=float(phi), apod_met=APOD_METHODS[apod_met],
               apod=ah, apod_par=0.0)  # win_par is not passed on (python/src/py_dream_arr_rect.cc:161-171)
    return _run(fn, Ro, c, device, arr)
