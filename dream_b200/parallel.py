"""Multi-GPU delay-and-sum over torch.distributed (NCCL between GPUs).

Frames are independent, so the common case needs no collective at all: each
rank beamforms its own frames (bench.py does this). A single frame larger than
one GPU's share can be split three ways:

* by transmit element (``das_shard_tx``): rank r holds only the A-scan columns of
  its block of outer elements (1/G of Y, the dominant array), beamforms a
  partial image over ALL pixels, and one all-reduce (SUM) of No image values
  adds the partial images. TFM only: RCA reads its stripe edges at fixed
  indices of the full element arrays (extra_src/das.cc:464-467), which a
  transmit subset would shift, so RCA frames use inner-element sharding.
* by inner element (``das_shard_inner``): rank r holds only the A-scan columns
  of its block of inner elements (TFM receivers, RCA col-tx rows, RCA row-tx
  columns) for every outer element, passes the FULL element arrays (so the RCA
  stripe edges are read where the reference reads them) and beamforms the
  partial image over its terms; one all-reduce adds them. This is how an RCA
  frame is split (268 MB of FP32 A-scans for the 128x128 array).
* by image point (``das_shard_pixels``): rank r beamforms a contiguous block of
  image points with the full Y and an all-gather assembles the image. Works for
  every method; every rank needs all of Y.

The adjoint splits the same way without a collective (``das_adjoint_shard_inner``):
the image-domain input is broadcast once and every rank writes the A-scan
columns of its own inner block.

The per-rank compute is a function argument so the sharding and collective
logic is the same whether a rank runs the CUDA kernels (``cuda_compute``) or,
in the CPU tests, the oracle.
"""
from __future__ import annotations

from typing import Callable

import numpy as np
import torch
import torch.distributed as dist


def block_range(n: int, world: int, rank: int):
    """Contiguous block [lo, hi) of n items for rank (sizes differ by at most 1)."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def tx_columns(method: str, Nt: int, Nr: int, o_lo: int, o_hi: int):
    """A-scan column range of transmit elements [o_lo, o_hi): TFM columns are
    t*Nr + r, so a block of transmit elements is contiguous."""
    if method != "tfm":
        raise ValueError("transmit sharding supports TFM (RCA: use das_shard_pixels)")
    return o_lo * Nr, o_hi * Nr


def das_shard_tx(compute: Callable, Y_local, Gt, Gr, Ro, dt, delay, cp, method, group=None):
    """Partial image over this rank's transmit block, summed over ranks.

    ``Y_local`` holds only this rank's A-scan columns (``tx_columns``). ``compute``
    is called as ``compute(Y_local, Gt_local, Gr, Ro, dt, delay, cp, method)`` and
    must return a 1-D torch tensor on the collective's device.
    """
    if method != "tfm":
        raise ValueError("transmit sharding supports TFM (RCA: use das_shard_pixels)")
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    lo, hi = block_range(int(Gt.shape[0]), world, rank)
    part = compute(Y_local, Gt[lo:hi], Gr, Ro, dt, delay, cp, method)
    dist.all_reduce(part, op=dist.ReduceOp.SUM, group=group)
    return part


def element_counts(method: str, Nt: int, Nr: int):
    """(outer, inner) element counts: RCA row-tx loops over rows (Gr) outside
    and columns (Gt) inside; TFM and RCA col-tx over Gt outside and Gr inside."""
    return (Nr, Nt) if method == "rca_rowtx" else (Nt, Nr)


def inner_columns(method: str, Nt: int, Nr: int, lo: int, hi: int) -> np.ndarray:
    """A-scan columns of inner elements [lo, hi) for every outer element, in
    the shard's order (column o * n_in + i of the full Y becomes column
    o * (hi - lo) + i - lo of the shard)."""
    if method == "saft":
        raise ValueError("SAFT has no inner elements to shard")
    n_out, n_in = element_counts(method, Nt, Nr)
    return (np.arange(n_out)[:, None] * n_in + np.arange(lo, hi)[None, :]).reshape(-1)


def das_shard_inner(compute: Callable, Y_local, Gt, Gr, Ro, dt, delay, cp, method, group=None):
    """Partial image over this rank's block of inner elements, summed over ranks.

    ``Y_local`` holds this rank's A-scan columns (``inner_columns``).
    ``compute(Y_local, Gt, Gr, Ro, dt, delay, cp, method, inner=(lo, hi))`` gets
    the full element arrays and must return the partial image as a 1-D torch
    tensor on the collective's device.
    """
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n_out, n_in = element_counts(method, int(Gt.shape[0]), int(Gr.shape[0]))
    lo, hi = block_range(n_in, world, rank)
    part = compute(Y_local, Gt, Gr, Ro, dt, delay, cp, method, inner=(lo, hi))
    dist.all_reduce(part, op=dist.ReduceOp.SUM, group=group)
    return part


def das_adjoint_shard_inner(compute_adjoint: Callable, x, Gt, Gr, Ro, dt, delay, cp, method, K, src=0,
                            group=None):
    """This rank's A-scan columns of the adjoint DAS^T x (no collective on the
    data path: x is broadcast from ``src`` once, then every rank writes the
    columns of its own block of inner elements).

    ``compute_adjoint(x, Gt, Gr, Ro, dt, delay, cp, method, K, inner=(lo, hi))``
    returns those columns as a K x (n_out * (hi - lo)) tensor.
    """
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dist.broadcast(x, src=src, group=group)
    n_out, n_in = element_counts(method, int(Gt.shape[0]), int(Gr.shape[0]))
    lo, hi = block_range(n_in, world, rank)
    return compute_adjoint(x, Gt, Gr, Ro, dt, delay, cp, method, K, inner=(lo, hi))


def das_shard_pixels(compute: Callable, Y, Gt, Gr, Ro, dt, delay, cp, method, group=None):
    """This rank's block of image points, all-gathered into the full image.

    ``compute(Y, Gt, Gr, Ro_block, dt, delay_block, cp, method)`` returns the
    block's 1-D image. Per-point sums are unchanged, so the assembled image
    equals the unsharded one exactly.
    """
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    No = int(Ro.shape[0])
    lo, hi = block_range(No, world, rank)
    d = delay if np.size(delay) == 1 else delay[lo:hi]
    part = compute(Y, Gt, Gr, Ro[lo:hi], dt, d, cp, method)
    sizes = [block_range(No, world, r) for r in range(world)]
    width = max(h - l for l, h in sizes)
    buf = torch.zeros(width, dtype=part.dtype, device=part.device)
    buf[: hi - lo] = part
    gathered = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(gathered, buf, group=group)
    return torch.cat([g[: h - l] for g, (l, h) in zip(gathered, sizes)])


def cuda_compute(storage: str = "f32", err_level: str = "ignore"):
    """Per-rank compute on the rank's GPU with the FP32/BF16-storage kernels."""
    from .beamformer import das_mixed

    def run(Y, Gt, Gr, Ro, dt, delay, cp, method, inner=None):
        dev = torch.device("cuda", torch.cuda.current_device())
        Yt = Y if (isinstance(Y, torch.Tensor) and Y.is_cuda) else torch.as_tensor(np.asarray(Y)).to(dev)
        return das_mixed(Yt, Gt, Gr, Ro, dt, delay, cp, method, err_level, f"cuda:{dev.index}", storage,
                         inner=inner)
    return run


def cuda_adjoint_compute():
    """Per-rank adjoint on the rank's GPU (the geometry-bound operator)."""
    from .autograd import DASOperator

    def run(x, Gt, Gr, Ro, dt, delay, cp, method, K, inner=None):
        dev = torch.device("cuda", torch.cuda.current_device())
        op = DASOperator(Gt, Gr, Ro, dt, delay, cp, method, K, device=dev, inner=inner)
        return op.adjoint(x.to(dev))
    return run
