"""Differentiable delay-and-sum: torch.autograd.Functions over the CUDA
operator, and the model-based least-squares (CG) reconstruction.

The reference has no adjoint; its model-based example builds an explicit DAS
matrix D and reconstructs with D' (examples/model_based_example.m:381-456).
Here the operator pair is matrix-free on the GPU, with w the per-A-scan
apodisation weights and k(n, c) the FP64 reference sample index:

    DAS_w  (gather):  Im[n]   = sum_c w[c] * Y[k(n,c), c]
    DAS_w^T (scatter): Ya[k, c] = w[c] * sum_{n: k(n,c)=k} x[n]

Both are exact adjoints of each other (same index set), so
<DAS_w Y, x> = <Y, DAS_w^T x> up to FP32 rounding.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .beamformer import _torch_fortran, grid_hint, parse_method


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class DASOperator:
    """Geometry-bound DAS operator on one CUDA device (FP32 samples).

    Ro, Gt, Gr, delay are kept on the device in FP64 (they are referenced by
    the bound plan); K is the A-scan length.
    """

    def __init__(self, Gt, Gr, Ro, dt, delay, cp, method, K, device="cuda", inner=None):
        self.device = torch.device(device) if not isinstance(device, torch.device) else device
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        das_type = parse_method(method)
        if das_type == _lib.SAFT:
            raise RuntimeError("DASOperator supports TFM and RCA methods")
        self.Gt = _torch_fortran(Gt, np.float64, self.device)
        self.Gr = _torch_fortran(Gr, np.float64, self.device)
        self.Ro = _torch_fortran(Ro, np.float64, self.device)
        self.delay = _torch_fortran(delay, np.float64, self.device)
        self.K = int(K)
        self.No = int(self.Ro.shape[0])
        self.Nt, self.Nr = int(self.Gt.shape[0]), int(self.Gr.shape[0])
        self.ncol = self.Nt * self.Nr
        self.inner = None
        if inner is not None:
            # an inner-element shard: the A-scans are the columns of inner elements [lo, hi)
            from .beamformer import inner_count
            lo, hi = int(inner[0]), int(inner[1])
            n_out, n_in = inner_count(das_type, self.Nt, self.Nr)
            if not (0 <= lo < hi <= n_in):
                raise RuntimeError("DASOperator: inner-element shard out of range")
            self.inner = (lo, hi)
            self.ncol = n_out * (hi - lo)
        multi = self.delay.numel() > 1
        if multi and self.delay.numel() != self.No:
            raise RuntimeError("Error in das!")
        self.plan = _lib.plan_create(das_type, self.K, self.No, self.Nt, self.Nr, _lib.PREC_F32_STORE,
                                     self.device.index)
        L = _lib.load()
        h = grid_hint(self.Ro)
        _lib.check(L.dream_das_set_grid_hint(self.plan.handle, h))
        if self.inner is not None:
            _lib.check(L.dream_das_set_inner_shard(self.plan.handle, *self.inner))
        self._L = L
        _lib.check(L.dream_das_bind_geometry(
            self.plan.handle, _p(self.Ro), _p(self.Gt), _p(self.Gr), float(dt),
            _lib.DELAY_MULTIPLE if multi else _lib.DELAY_SINGLE, _p(self.delay), float(cp),
            self._stream()))
        self.d_oob = torch.zeros(1, dtype=torch.int64, device=self.device)

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _ascans(self, Y):
        """Y as FP32 column-major (K, ncol) on the device."""
        Y = _torch_fortran(Y, np.float32, self.device)
        if tuple(Y.shape) != (self.K, self.ncol):
            raise RuntimeError(f"A-scans must be {self.K} x {self.ncol}")
        return Y

    def _weights(self, w):
        if w is None:
            return None
        w = w.to(device=self.device, dtype=torch.float32).reshape(-1).contiguous()
        if w.numel() != self.ncol:
            raise RuntimeError(f"weights need {self.ncol} values")
        return w

    def forward(self, Y, w=None):
        """DAS_w Y -> image (No,) FP32."""
        Y = self._ascans(Y)
        w = self._weights(w)
        Im = torch.empty(self.No, dtype=torch.float32, device=self.device)
        _lib.check(self._L.dream_das_op_forward(self.plan.handle, _p(Y), _p(w), _p(Im), _p(self.d_oob),
                                                self._stream()))
        return Im

    def adjoint(self, x, w=None):
        """DAS_w^T x -> A-scans (K, ncol) FP32, column-major storage."""
        x = x.to(device=self.device, dtype=torch.float32).reshape(-1).contiguous()
        w = self._weights(w)
        Ya = torch.empty((self.ncol, self.K), dtype=torch.float32, device=self.device)
        _lib.check(self._L.dream_das_op_adjoint(self.plan.handle, _p(x), _p(w), _p(Ya), self._stream()))
        return Ya.t()

    def wgrad(self, g, Y):
        """dW[c] = sum_n g[n] Y[k(n,c), c]."""
        g = g.to(device=self.device, dtype=torch.float32).reshape(-1).contiguous()
        Y = self._ascans(Y)
        dW = torch.empty(self.ncol, dtype=torch.float32, device=self.device)
        _lib.check(self._L.dream_das_op_wgrad(self.plan.handle, _p(g), _p(Y), _p(dW), self._stream()))
        return dW

    def backward(self, g, Y, w=None):
        """(DAS_w^T g, wgrad(g, Y)) in one pass."""
        g = g.to(device=self.device, dtype=torch.float32).reshape(-1).contiguous()
        Y = self._ascans(Y)
        w = self._weights(w)
        Yg = torch.empty((self.ncol, self.K), dtype=torch.float32, device=self.device)
        dW = torch.empty(self.ncol, dtype=torch.float32, device=self.device)
        _lib.check(self._L.dream_das_op_backward(self.plan.handle, _p(g), _p(Y), _p(w), _p(Yg), _p(dW),
                                                 self._stream()))
        return Yg.t(), dW

    def oob_count(self) -> int:
        return int(self.d_oob.item())


class DASGather(torch.autograd.Function):
    """Im = DAS_w(Y); differentiable in Y and w."""

    @staticmethod
    def forward(ctx, Y, w, op):
        ctx.op = op
        ctx.save_for_backward(Y, w)
        return op.forward(Y, w)

    @staticmethod
    def backward(ctx, g):
        Y, w = ctx.saved_tensors
        op = ctx.op
        gY = gw = None
        if ctx.needs_input_grad[0] and ctx.needs_input_grad[1]:
            gY, gw = op.backward(g, Y, w)
        elif ctx.needs_input_grad[0]:
            gY = op.adjoint(g, w)
        elif ctx.needs_input_grad[1]:
            gw = op.wgrad(g, Y)
        if gY is not None:
            gY = gY.to(Y.dtype)
        if gw is not None:
            gw = gw.to(w.dtype).reshape(w.shape)
        return gY, gw, None


class DASScatter(torch.autograd.Function):
    """Y = DAS_w^T(x) (A-scans synthesised from an image); differentiable in x and w."""

    @staticmethod
    def forward(ctx, x, w, op):
        ctx.op = op
        ctx.save_for_backward(x, w)
        return op.adjoint(x, w)

    @staticmethod
    def backward(ctx, R):
        x, w = ctx.saved_tensors
        op = ctx.op
        gx = gw = None
        if ctx.needs_input_grad[0]:
            gx = op.forward(R, w).to(x.dtype).reshape(x.shape)
        if ctx.needs_input_grad[1]:
            gw = op.wgrad(x, R).to(w.dtype).reshape(w.shape)
        return gx, gw, None


def das_gather(Y, w, op):
    return DASGather.apply(Y, w, op)


def das_scatter(x, w, op):
    return DASScatter.apply(x, w, op)


def cg_reconstruct(op: DASOperator, Y, w, lam: float = 1e-3, iters: int = 30, x0=None):
    """Solves min_x ||DAS_w^T x - Y||^2 + lam ||x||^2 with conjugate gradients
    on the normal equations (DAS_w DAS_w^T + lam I) x = DAS_w Y.

    Each iteration applies the scatter and the gather once. Returns
    (x, residual norms per iteration).
    """
    Y = op._ascans(Y)
    b = op.forward(Y, w)
    x = torch.zeros_like(b) if x0 is None else x0.clone()
    r = b - (op.forward(op.adjoint(x, w), w) + lam * x) if x0 is not None else b.clone()
    p = r.clone()
    rs = torch.dot(r, r)
    hist = []
    for _ in range(iters):
        Ap = op.forward(op.adjoint(p, w), w) + lam * p
        alpha = rs / torch.dot(p, Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        rs_new = torch.dot(r, r)
        hist.append(rs_new)
        p = r + (rs_new / rs) * p
        rs = rs_new
    return x, torch.stack(hist).sqrt() if hist else torch.zeros(0, device=b.device)


class CGGraph:
    """``cg_reconstruct`` captured once in a CUDA graph.

    ``Y`` and ``w`` are copied into static buffers (``self.Y``, ``self.w``);
    write new A-scans or weights into them and call ``replay()`` to solve
    again without any host-side launch overhead. ``self.x`` and
    ``self.residuals`` hold the latest solution.
    """

    def __init__(self, op: DASOperator, Y, w, lam: float = 1e-3, iters: int = 30):
        self.op = op
        self.Y = op._ascans(Y).clone()
        self.w = w.to(device=op.device, dtype=torch.float32).clone()
        side = torch.cuda.Stream(op.device)
        side.wait_stream(torch.cuda.current_stream(op.device))
        with torch.cuda.stream(side):
            cg_reconstruct(op, self.Y, self.w, lam, 2)  # warm-up outside the capture
        torch.cuda.current_stream(op.device).wait_stream(side)
        torch.cuda.synchronize(op.device)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.x, self.residuals = cg_reconstruct(op, self.Y, self.w, lam, iters)

    def replay(self):
        self.graph.replay()
        return self.x, self.residuals
