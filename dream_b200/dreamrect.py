"""``dreamrect`` on the GPU: the spatial impulse response of a rectangular
transducer, the CUDA counterpart of the reference module ``dreamrect``
(python/src/py_dreamrect.cc:47-139; src/dreamrect.cc, opencl/dreamrect.cl).

    H = dreamrect(Ro, geom_par, s_par, delay, m_par, err_level="stop", device="cuda")

Ro: No x 3 observation points (mm). geom_par = [a, b]: element size (mm).
s_par = [dx, dy, dt, nt]: surface discretisation (mm), sampling period (us),
SIR length. delay (us): a scalar or one value per point. m_par = [v, cp,
alpha]: normal velocity, sound speed (m/s), attenuation (only alpha = 0: the
reference's attenuation filter has no CUDA counterpart). Returns H, nt x No
FP64 column-major (a CUDA tensor when Ro is one), equal to the reference's
bit for bit. err_level 'ignore' / 'warn' / 'stop' treats samples outside
[0, nt) as the reference does ('stop' raises).
"""
from __future__ import annotations

import ctypes
import sys

import numpy as np

from . import _lib
from .beamformer import _is_torch, parse_device, parse_err_level


def _fail(msg):
    sys.stderr.write(msg + "\n")
    raise RuntimeError("Error in dreamrect!")


def _vector(p, n, what):
    a = np.asarray(p.cpu() if _is_torch(p) else p, dtype=np.float64)
    if not (a.size == n and (a.ndim <= 1 or (a.ndim == 2 and 1 in a.shape))):
        _fail(f"dreamrect requires that {what} must be a {n} element vector!")
    return a.reshape(-1)


def dreamrect(Ro, geom_par, s_par, delay, m_par, err_level="stop", device="cuda"):
    on_device = _is_torch(Ro) and Ro.device.type == "cuda"
    shape = tuple(Ro.shape)
    if len(shape) != 2 or shape[1] != 3:
        _fail("dreamrect requires that observation point arg must be a (number of observation points) x 3 matrix!")
    No = shape[0]
    a, b = _vector(geom_par, 2, "the geometry arg")
    dx, dy, dt, nt_f = _vector(s_par, 4, "sampling par arg")
    nt = int(nt_f)
    v, cp, alpha = _vector(m_par, 3, "material parameters par arg")
    if alpha > np.finfo(np.float64).eps:
        raise RuntimeError("dreamrect: attenuation (alpha > 0) is not supported by the CUDA backend")
    d = np.asarray(delay.cpu() if _is_torch(delay) else delay, dtype=np.float64)
    if d.size > 1 and (d.size != No or not (d.ndim <= 1 or 1 in d.shape)):
        _fail(f"dreamrect requires that delay arg must be a {d.size} element vector (with a length equal to "
              "the number of observation points) or a scalar!")
    if d.size < 1:
        _fail("dreamrect requires a delay")
    level = parse_err_level(err_level)
    multi = _lib.DELAY_MULTIPLE if d.size > 1 else _lib.DELAY_SINGLE
    L = _lib.load()
    oob = ctypes.c_int64(0)
    if on_device:
        import torch
        dev = Ro.device
        Rt = Ro.to(torch.float64).t().contiguous().t()
        dt_ = torch.as_tensor(d.reshape(-1), device=dev)
        H = torch.empty((No, nt), dtype=torch.float64, device=dev).t()
        p = lambda t: ctypes.c_void_p(t.data_ptr()) if t.numel() else None
        st = L.dream_rect_run_device(p(Rt), No, a, b, dx, dy, dt, nt, multi, p(dt_), v, cp, p(H), level,
                                     ctypes.byref(oob), dev.index if dev.index is not None else 0,
                                     ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    else:
        Rh = np.asfortranarray(np.asarray(Ro, dtype=np.float64))
        dh = np.ascontiguousarray(d.reshape(-1))
        H = np.zeros((nt, No), dtype=np.float64, order="F")
        p = lambda x: x.ctypes.data_as(ctypes.c_void_p) if x.size else None
        st = L.dream_rect_run(p(Rh), No, a, b, dx, dy, dt, nt, multi, p(dh), v, cp, p(H), level, ctypes.byref(oob),
                              parse_device(device))
    _lib.check(st)
    if st == _lib.STATUS_OOB:
        _fail("SIR out-of-bounds!")
    if st == _lib.STATUS_WARN_OOB:
        print("Warning: SIR out-of-bounds!")
    return H
