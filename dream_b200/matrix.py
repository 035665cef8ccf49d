"""The delay-and-sum beamformer as an explicit sparse matrix, for
model-based reconstruction (the reference builds it densely in
examples/model_based_example.m:381-456, with a stale ``das`` interface).

    idx = das_indices(Gt, Gr, Ro, dt, delay, cp, method, K)      # (terms, No) int64
    D   = das_matrix(Gt, Gr, Ro, dt, delay, cp, method, K)       # (No, K*terms) CSR

``idx[c, n]`` is the sample of A-scan column c that ``das`` adds for image
point n, or -1 for an out-of-bounds term. ``D`` has the entry 1 (or
``weights[c]``) at (n, c*K + idx[c, n]), so with the A-scans flattened
column-major, ``D @ Y.reshape(-1, order='F')`` is the beamformed image (for
FP64 and unit weights it equals ``das`` bit for bit when each row is summed
in column order), ``D.T`` is the adjoint, and ``D`` can be handed to any
sparse solver. ``precision='f64'`` gives the indices of ``das`` (and of the
FP32/BF16-storage kernels), ``'f32'`` those of ``das_f``.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .beamformer import _check_shapes, _torch_fortran, parse_device, parse_method


def das_indices(Gt, Gr, Ro, dt, delay, cp, method, K, precision="f64", device="cuda"):
    """Per-term sample indices (terms x No, int64 CUDA tensor, -1 out of
    bounds) and the out-of-bounds count."""
    das_type = parse_method(method)
    dev = torch.device("cuda", parse_device(device)) if not isinstance(device, torch.device) else device
    gdt = np.float32 if precision == "f32" else np.float64
    Gt_t = _torch_fortran(Gt, gdt, dev)
    Gr_t = _torch_fortran(Gr, gdt, dev) if Gr is not None and das_type != _lib.SAFT else None
    Ro_t = _torch_fortran(Ro, gdt, dev)
    dl_t = _torch_fortran(delay, gdt, dev)
    No, Nt, Nr, multi = _shapes(Gt_t, Gr_t, Ro_t, dl_t, das_type)
    eff_saft = das_type == _lib.SAFT or Nr == 0
    terms = Nt if eff_saft else Nt * Nr
    prec = _lib.PREC_F32 if precision == "f32" else _lib.PREC_F64
    plan = _lib.plan_create(das_type, int(K), No, Nt, 0 if eff_saft else Nr, prec, dev.index)
    idx = torch.empty((terms, No), dtype=torch.int64, device=dev)
    oob = ctypes.c_int64(0)
    p = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() else None
    _lib.check(_lib.load().dream_das_indices_device(
        plan.handle, p(Ro_t), p(Gt_t), p(Gr_t), float(dt), _lib.DELAY_MULTIPLE if multi else _lib.DELAY_SINGLE,
        p(dl_t), float(cp), p(idx), ctypes.byref(oob), ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
    return idx, int(oob.value)


def _shapes(Gt, Gr, Ro, dl, das_type):
    """(No, Nt, Nr, multi) with the reference binding's shape checks."""
    Nt = int(Gt.shape[0])
    Nr = int(Gr.shape[0]) if Gr is not None else 0
    ascans = np.zeros((1, Nt * max(Nr, 1)))  # shape only: every column the method reads
    _, No, Nt, Nr, multi = _check_shapes(ascans, Gt, Gr, Ro, dl, das_type)
    return No, Nt, Nr, multi


def das_matrix(Gt, Gr, Ro, dt, delay, cp, method, K, weights=None, precision="f64", device="cuda",
               dtype=torch.float64):
    """The beamformer as a CSR matrix (No x K*terms) on the device: row n
    holds weights[c] (or 1) at column c*K + idx[c, n] for every in-bounds
    term, in increasing column order."""
    idx, _ = das_indices(Gt, Gr, Ro, dt, delay, cp, method, K, precision, device)
    terms, No = idx.shape
    it = idx.t()  # (No, terms): row-major traversal gives (point, column) in CSR order
    valid = it >= 0
    counts = valid.sum(1)
    crow = torch.zeros(No + 1, dtype=torch.int64, device=idx.device)
    torch.cumsum(counts, 0, out=crow[1:])
    n_idx, c_idx = valid.nonzero(as_tuple=True)
    cols = c_idx * int(K) + it[n_idx, c_idx]
    if weights is None:
        vals = torch.ones(cols.numel(), dtype=dtype, device=idx.device)
    else:
        w = torch.as_tensor(weights, dtype=dtype, device=idx.device).reshape(-1)
        if w.numel() != terms:
            raise RuntimeError(f"das_matrix: weights need {terms} values (one per A-scan column)")
        vals = w[c_idx]
    return torch.sparse_csr_tensor(crow, cols, vals, size=(No, int(K) * terms))
