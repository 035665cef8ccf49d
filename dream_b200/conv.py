"""Column-wise convolution on the GPU: the CUDA counterparts of DREAM's
``fftconv_p`` (python/src/py_fftconv_p.cc, python/include/py_fftconv_p.hpp)
and ``conv_p`` (extra_src/oct_conv_p.cc), which turn spatial impulse
responses into the A-scans that ``das`` beamforms.

    Y = fftconv_p(A, B)                 # Y[:, n] = A[:, n] * B[:, n] or A[:, n] * B
    Y = conv_p(A, B)
    conv_p(A, B, Y, mode)               # in place: mode '=', '+=' or '-='

A is A_M x A_N; B a vector (either orientation) used for every column, or an
A_M' x A_N matrix; Y has A_M + B_M - 1 rows. FP64, column-major (F-order
NumPy arrays, or CUDA tensors whose transposes are contiguous). Every output
sums its products in the order of the reference's direct conv()
(extra_src/conv.cc:34-78) without fused multiply-add, so it equals conv() bit
for bit and FFTW's fftconv_p to rounding. NumPy inputs are processed through
the host entry of the C ABI (dream_conv_p_run); CUDA tensors stay on their
device (dream_conv_p_run_device on the current stream).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .beamformer import _is_torch, parse_device

_MODES = {"=": _lib.CONV_EQU, "+=": _lib.CONV_SUM, "-=": _lib.CONV_NEG}


def _dims(a):
    s = tuple(a.shape)
    if len(s) == 0:
        return 1, 1
    if len(s) == 1:
        return s[0], 1
    if len(s) == 2:
        return s[0], s[1]
    raise RuntimeError("arguments must be vectors or matrices")


def _device_fortran(t):
    import torch
    t = t.to(torch.float64)
    if t.dim() == 1:
        t = t.reshape(-1, 1)
    return t.t().contiguous().t()


def _run(A, B, Y, mode_code, device):
    if _is_torch(A) and A.device.type == "cuda":
        import torch
        Ad = _device_fortran(A)
        Bd = _device_fortran(B.to(A.device) if _is_torch(B) else torch.as_tensor(np.asarray(B), device=A.device))
        A_M, A_N = _dims(Ad)
        B_M, B_N = _dims(Bd)
        if B_M != 1 and B_N != 1 and B_N != A_N:
            raise RuntimeError("Argument 2 must be a vector or a matrix with the same number of columns as arg 1!")
        Lb = B_M * B_N if (B_M == 1 or B_N == 1) else B_M
        if Y is None:
            Y = torch.empty((A_N, A_M + Lb - 1), dtype=torch.float64, device=A.device).t()  # column-major
        p = lambda t: ctypes.c_void_p(t.data_ptr()) if t.numel() else None
        st = ctypes.c_void_p(torch.cuda.current_stream(A.device).cuda_stream)
        _lib.check(_lib.load().dream_conv_p_run_device(p(Ad), A_M, A_N, p(Bd), B_M, B_N, p(Y), mode_code, st))
        return Y
    dev = parse_device(device)
    Ah = np.asfortranarray(np.asarray(A.cpu() if _is_torch(A) else A, dtype=np.float64))
    Bh = np.asfortranarray(np.asarray(B.cpu() if _is_torch(B) else B, dtype=np.float64))
    A_M, A_N = _dims(Ah)
    B_M, B_N = _dims(Bh)
    if B_M != 1 and B_N != 1 and B_N != A_N:
        raise RuntimeError("Argument 2 must be a vector or a matrix with the same number of columns as arg 1!")
    Lb = B_M * B_N if (B_M == 1 or B_N == 1) else B_M
    if Y is None:
        Y = np.empty((A_M + Lb - 1, A_N), dtype=np.float64, order="F")
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p) if a.size else None
    _lib.check(_lib.load().dream_conv_p_run(p(Ah), A_M, A_N, p(Bh), B_M, B_N, p(Y), mode_code, dev))
    return Y


def fftconv_p(A, B, device="cuda"):
    """``Y = fftconv_p(A, B)``: full linear convolution of every column of A
    with B (a vector, or the matching column of a matrix)."""
    return _run(A, B, None, _lib.CONV_EQU, device)


def conv_p(A, B, Y=None, mode="=", device="cuda"):
    """``Y = conv_p(A, B)`` or, with Y given, ``conv_p(A, B, Y, mode)`` updating
    Y in place ('=' replace, '+=' add, '-=' subtract); returns Y.

    Y must then have A_M + B_M - 1 rows and A_N columns: an F-order FP64
    NumPy array, or an FP64 CUDA tensor with column-major storage."""
    if mode not in _MODES:
        raise RuntimeError("Non-valid string in arg 4!")
    if Y is None:
        return _run(A, B, None, _MODES[mode], device)
    A_M, A_N = _dims(A)
    B_M, B_N = _dims(B)
    Lb = B_M * B_N if (B_M == 1 or B_N == 1) else B_M
    if _dims(Y)[0] != A_M + Lb - 1:
        raise RuntimeError("Wrong number of rows in argument 3!")
    if _dims(Y)[1] != A_N:
        raise RuntimeError("Wrong number of columns in argument 3!")
    if _is_torch(Y):
        import torch
        if not (Y.is_cuda and Y.dtype == torch.float64 and Y.dim() == 2 and Y.stride(0) == 1):
            raise RuntimeError("conv_p: Y must be a column-major FP64 CUDA tensor")
        if not (_is_torch(A) and A.is_cuda):
            A = torch.as_tensor(np.asarray(A, dtype=np.float64), device=Y.device)
    elif not (isinstance(Y, np.ndarray) and Y.dtype == np.float64 and Y.flags["F_CONTIGUOUS"]):
        raise RuntimeError("conv_p: Y must be an F-order float64 array")
    return _run(A, B, Y, _MODES[mode], device)


def fmc_synthesis(Ht, pulse, Hr=None, device="cuda"):
    """Full-matrix-capture A-scans from element SIRs in two launches: column
    ``t*L_r + r`` is ``(Hr[:, r] (*) Ht[:, t]) (*) pulse``, which the
    reference's tests build with two fftconv_p calls per transmit
    (python/tests/test_das_tfm.py:110-115, with Hr = Ht; test_das_rca.py:117-124).
    Ht: M x L_t transmit SIRs, Hr: M x L_r receive SIRs (default Ht), pulse:
    P_M samples. Returns (2M-1 + P_M-1) x L_t*L_r FP64 (column-major), equal
    to the per-transmit calls bit for bit: a CUDA tensor when Ht is one, else
    a NumPy array."""
    import torch
    on_device = _is_torch(Ht) and Ht.device.type == "cuda"
    dev = Ht.device if on_device else torch.device("cuda", parse_device(device))
    as_dev = lambda a: _device_fortran(a.to(dev) if _is_torch(a) else torch.as_tensor(np.asarray(a), device=dev))
    Htd = as_dev(Ht)
    Hrd = Htd if Hr is None else as_dev(Hr)
    Pd = as_dev(pulse).reshape(-1).contiguous()
    M, L_t = _dims(Htd)
    M_r, L_r = _dims(Hrd)
    if M_r != M:
        raise RuntimeError("fmc_synthesis: the transmit and receive SIRs must have the same length")
    P_M = Pd.numel()
    N = L_t * L_r
    DP = torch.empty((N, 2 * M - 1), dtype=torch.float64, device=dev).t()
    Y = torch.empty((N, 2 * M - 1 + P_M - 1), dtype=torch.float64, device=dev).t()
    p = lambda t: ctypes.c_void_p(t.data_ptr()) if t.numel() else None
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(_lib.load().dream_conv_p_fmc_device(p(Htd), M, L_t, p(Hrd), L_r, p(Pd), P_M, p(DP), p(Y), st))
    del DP  # stream-ordered release: the caching allocator reuses it only after the launches
    return Y if on_device else Y.cpu().numpy()
