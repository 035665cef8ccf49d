"""Batched DAS: many frames of uneven shapes in one persistent launch, with an
optional CUDA graph around it (dream_das_batch_* in include/dream_das.h).

Each frame is one TFM/RCA beamforming problem on the device: FP32 (or BF16)
A-scans, FP64 geometry, FP32 image. Tile shapes and inner-chunk lengths come
from the autotuner (dream_b200.autotune) unless given per frame.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from . import _lib
from .beamformer import _torch_fortran, grid_hint, parse_method


class FrameStruct(ctypes.Structure):
    """Mirror of ``dream_das_frame``."""

    _fields_ = [
        ("das_type", ctypes.c_int),
        ("a_scan_len", ctypes.c_int64),
        ("No", ctypes.c_int64),
        ("num_t_elements", ctypes.c_int64),
        ("num_r_elements", ctypes.c_int64),
        ("Y", ctypes.c_void_p),
        ("Ro", ctypes.c_void_p),
        ("Gt", ctypes.c_void_p),
        ("Gr", ctypes.c_void_p),
        ("delay", ctypes.c_void_p),
        ("delay_type", ctypes.c_int),
        ("dt", ctypes.c_double),
        ("cp", ctypes.c_double),
        ("Im", ctypes.c_void_p),
        ("n_fast", ctypes.c_int64),
        ("tile_f", ctypes.c_int),
        ("tile_s", ctypes.c_int),
        ("jc", ctypes.c_int),
    ]


def _lib_batch():
    return _lib.load()


@dataclass
class Frame:
    """One frame on the device (geometry FP64, A-scans FP32 or BF16)."""

    Y: torch.Tensor
    Gt: torch.Tensor
    Gr: torch.Tensor
    Ro: torch.Tensor
    delay: torch.Tensor
    dt: float
    cp: float
    method: str = "tfm"
    Im: Optional[torch.Tensor] = None
    n_fast: int = -1
    tile: Optional[tuple] = None
    jc: int = 0

    @property
    def sums(self) -> int:
        return int(self.Ro.shape[0]) * int(self.Gt.shape[0]) * int(self.Gr.shape[0])


def make_frame(Y, Gt, Gr, Ro, dt, delay, cp, method="tfm", device="cuda", storage="f32") -> Frame:
    dev = torch.device(device)
    Yt = _torch_fortran(Y, np.float32, dev)
    if storage == "bf16":
        Yt = Yt.t().contiguous().to(torch.bfloat16).t()
    f = Frame(Yt, _torch_fortran(Gt, np.float64, dev), _torch_fortran(Gr, np.float64, dev),
              _torch_fortran(Ro, np.float64, dev), _torch_fortran(delay, np.float64, dev), float(dt), float(cp),
              method)
    f.Im = torch.empty(int(f.Ro.shape[0]), dtype=torch.float32, device=dev)
    return f


class DASBatch:
    """A fixed set of frames beamformed by one persistent kernel launch."""

    def __init__(self, frames, storage="f32", device=None, autotune=True):
        self.frames = list(frames)
        self.storage = storage
        dev = self.frames[0].Y.device if self.frames else torch.device("cuda")
        self.device = dev
        L = _lib_batch()
        self._L = L
        if autotune:
            from .autotune import batch_config
            for f in self.frames:
                if f.n_fast < 0:
                    f.n_fast = grid_hint(f.Ro)  # always the frame's own grid
                if f.tile is None or not f.jc:
                    cfg = batch_config(f, storage)  # shared by the frames of a bucket
                    if (cfg["n_fast"] > 0) == (f.n_fast > 0):
                        f.tile = f.tile or tuple(cfg["tile"])
                        f.jc = f.jc or cfg["jc"]
        arr = (FrameStruct * max(1, len(self.frames)))()
        for i, f in enumerate(self.frames):
            if f.n_fast < 0:
                f.n_fast = grid_hint(f.Ro)
            t = f.tile or (0, 0)
            arr[i] = FrameStruct(
                parse_method(f.method), int(f.Y.shape[0]), int(f.Ro.shape[0]), int(f.Gt.shape[0]),
                int(f.Gr.shape[0]), f.Y.data_ptr(), f.Ro.data_ptr(), f.Gt.data_ptr(), f.Gr.data_ptr(),
                f.delay.data_ptr(), _lib.DELAY_MULTIPLE if f.delay.numel() > 1 else _lib.DELAY_SINGLE,
                f.dt, f.cp, f.Im.data_ptr(), int(f.n_fast), int(t[0]), int(t[1]), int(f.jc))
        self._arr = arr
        h = ctypes.c_void_p()
        prec = _lib.PREC_BF16_STORE if storage == "bf16" else _lib.PREC_F32_STORE
        idx = dev.index if dev.index is not None else torch.cuda.current_device()
        _lib.check(L.dream_das_batch_create(ctypes.byref(h), ctypes.cast(arr, ctypes.c_void_p), len(self.frames),
                                            prec, idx))
        self.handle = h
        self.d_oob = torch.zeros(1, dtype=torch.int64, device=dev)
        self.graph = None

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self._L.dream_das_batch_destroy(h)
            self.handle = None

    @property
    def sums(self) -> int:
        return sum(f.sums for f in self.frames)

    @property
    def items(self) -> int:
        return int(self._L.dream_das_batch_items(self.handle))

    @property
    def grid(self) -> int:
        return int(self._L.dream_das_batch_grid(self.handle))

    def run(self):
        """One persistent launch on the current stream (asynchronous)."""
        s = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._L.dream_das_batch_run(self.handle, ctypes.c_void_p(self.d_oob.data_ptr()),
                                               ctypes.c_void_p(s)))

    def capture(self) -> torch.cuda.CUDAGraph:
        """Captures run() in a CUDA graph (replay with self.graph.replay())."""
        self.run()  # uploads the frame table outside the capture
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.run()
        torch.cuda.current_stream(self.device).wait_stream(s)
        self.graph = g
        return g

    def oob_count(self) -> int:
        return int(self.d_oob.item())
