"""Autotuner for the FP32/BF16-storage DAS kernels.

Picks, per shape bucket, the CTA tile of image points (tile_f x tile_s) and
the inner-chunk length (8 or 16 register-resident legs) by timing each
candidate on the actual frame with CUDA events (median of a few runs after a
warm-up, the L2 cache flushed before each timed run: a frame that arrives from
the host or from another kernel is not L2-resident, and shapes that win with
warm caches can lose without them). Results are cached in a JSON file keyed by GPU name, method,
storage and bucket, so later processes reuse them:

    $DREAM_AUTOTUNE_CACHE or ~/.cache/dream_b200/autotune.json

Buckets: element counts exactly, A-scan length and grid extents rounded up to
powers of two (the kernels' cost depends on them smoothly).
"""
from __future__ import annotations

import ctypes
import json
import os
import threading

import torch

from . import _lib
from .beamformer import grid_hint, parse_method

_lock = threading.Lock()
_mem = None


def cache_path() -> str:
    return os.environ.get("DREAM_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "dream_b200", "autotune.json"))


def _load():
    global _mem
    if _mem is None:
        try:
            with open(cache_path()) as f:
                _mem = json.load(f)
        except Exception:
            _mem = {}
    return _mem


def _save():
    p = cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = p + f".{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(_mem, f, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except OSError:
        pass  # a read-only cache location only costs re-tuning


def _p2(n: int) -> int:
    n = max(1, int(n))
    return 1 << (n - 1).bit_length()


def bucket_key(method, storage, Nt, Nr, K, n_fast, No, nthr, device) -> str:
    name = torch.cuda.get_device_name(device).replace(" ", "_")
    n_slow = No // n_fast if n_fast else 1
    return (f"v2|{name}|{method}|{storage}|nthr={nthr}|Nt={Nt}|Nr={Nr}|K={_p2(K)}|"
            f"grid={_p2(n_fast) if n_fast else 0}x{_p2(n_slow)}")


def candidates(hinted: bool, nthr: int):
    """(tile_f, tile_s, jc) shapes with tile_f*tile_s == nthr."""
    out = []
    if hinted:
        for tf in (8, 16, 32, 64):
            ts = nthr // tf
            if ts >= 4 and ts % 4 == 0 and tf * ts == nthr:
                out += [(tf, ts, 16), (tf, ts, 8)]
    else:
        out += [(nthr, 1, 16), (nthr, 1, 8)]
    return out


L2_FLUSH_BYTES = 192 << 20  # more than the 126 MB L2


def _time_plan(plan_handle, args, flush, reps=5):
    L = _lib.load()
    st = torch.cuda.current_stream()
    L.dream_das_run_device_async(*args)  # warm-up
    ts = []
    for r in range(reps):
        flush.fill_(float(r))  # evicts the A-scans from L2
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        _lib.check(L.dream_das_run_device_async(*args))
        b.record(st)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    ts.sort()
    return ts[len(ts) // 2]


def tune(Y, Gt, Gr, Ro, dt, delay, cp, method="tfm", storage="f32", nthr=None, force=False):
    """Best {tile, jc, n_fast, ms} for this frame's bucket (cached).

    Y (FP32, or BF16 for storage 'bf16'), Gt, Gr, Ro, delay are column-major
    device tensors as the C ABI takes them. nthr=128 restricts the search to
    the persistent batch kernel's CTA size; None also tries 256-point tiles.
    """
    das_type = parse_method(method)
    dev = Y.device
    K, No, Nt, Nr = int(Y.shape[0]), int(Ro.shape[0]), int(Gt.shape[0]), int(Gr.shape[0])
    n_fast = grid_hint(Ro)
    key = bucket_key(method, storage, Nt, Nr, K, n_fast, No, nthr or 0, dev)
    with _lock:
        cache = _load()
        if not force and key in cache:
            return dict(cache[key])
    prec = _lib.PREC_BF16_STORE if storage == "bf16" else _lib.PREC_F32_STORE
    plan = _lib.plan_create(das_type, K, No, Nt, Nr, prec, dev.index if dev.index is not None else 0)
    L = _lib.load()
    _lib.check(L.dream_das_set_grid_hint(plan.handle, n_fast))
    Im = torch.empty(No, dtype=torch.float32, device=dev)
    d_oob = torch.zeros(1, dtype=torch.int64, device=dev)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    args = (plan.handle, ptr(Y), ptr(Ro), ptr(Gt), ptr(Gr), float(dt),
            _lib.DELAY_MULTIPLE if delay.numel() > 1 else _lib.DELAY_SINGLE, ptr(delay), float(cp), ptr(Im),
            ptr(d_oob), ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    sizes = [nthr] if nthr else [128, 256]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    best = None
    for n in sizes:
        for tf, ts, jc in candidates(n_fast > 0, n):
            if L.dream_das_set_tile(plan.handle, tf, ts) != 0:
                continue
            _lib.check(L.dream_das_set_chunk(plan.handle, jc))
            ms = _time_plan(plan.handle, args, flush)
            if best is None or ms < best["ms"]:
                best = {"tile": [tf, ts], "jc": jc, "n_fast": n_fast, "ms": ms}
    del flush
    with _lock:
        _load()[key] = best
        _save()
    return dict(best)


def apply(plan, cfg, Ro) -> None:
    """Sets a tuned configuration on a plan. The grid hint is taken from the
    plan's own image points Ro (a cached entry is shared by every grid of its
    bucket); the tile applies when the hinted/unhinted kind matches."""
    L = _lib.load()
    h = grid_hint(Ro)
    _lib.check(L.dream_das_set_grid_hint(plan.handle, h))
    if (h > 0) == (int(cfg["n_fast"]) > 0):
        _lib.check(L.dream_das_set_tile(plan.handle, int(cfg["tile"][0]), int(cfg["tile"][1])))
    _lib.check(L.dream_das_set_chunk(plan.handle, int(cfg["jc"])))


def batch_config(frame, storage="f32"):
    """Tuned 128-point tile and chunk for one batch frame (dream_b200.batch.Frame)."""
    return tune(frame.Y, frame.Gt, frame.Gr, frame.Ro, frame.dt, frame.delay, frame.cp, frame.method, storage,
                nthr=128)
