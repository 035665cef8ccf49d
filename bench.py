#!/usr/bin/env python
"""DAS beamformer benchmark on B200: pixel x tx x rx sums per second.

Workload (one "step"): one delay-and-sum frame of the TFM full-matrix-capture
configuration -- 64 x 64 elements (pitch 0.5 mm), K = 3000 samples
(dt = 0.04 us, cp = 1500 m/s), 512 x 512 image (x in [-20, 20] mm,
z in [2, 50] mm) = 1.074e9 sums -- on seeded synthetic A-scans.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Each rank beamforms its own frame (frames are independent: weak scaling, no
data-path collective). One JSON line is printed by rank 0.

value : whole-job Gsum/s with inputs resident in HBM (CUDA events on the
        launching stream, L2 flushed between steps by writing 256 MiB).
e2e   : the same metric through the public API (dream_b200.beamformer.das_mixed) from
        pinned host arrays: H2D of the inputs and D2H of the image each step.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DAS Gsum/s (pixel x tx x rx); adjoint-CG ms in adjoint_cg"
WORKLOAD = "TFM FMC 64x64 elements, K=3000, 512x512 image"
FALLBACK_HBM_GBS = 6650.0


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def make_scene(rank: int):
    from dream_b200 import synth
    return synth.tfm_scene(seed=1 + rank)


def cpu_baseline(scene, budget_s: float = 20.0):
    """The reference das_f (built from the reference sources into oracle/_ref)
    on the host cores; falls back to the C restatement (single thread) on a
    pixel sample when the reference build is absent."""
    from oracle import oracle
    nproc = os.cpu_count() or 1
    os.environ["DREAM_NUM_THREADS"] = str(nproc)
    s = scene.astype(np.float32)
    mod = oracle.reference_module("f32")
    if mod is not None:
        best, runs, t_all = None, 0, time.perf_counter()
        while runs < 3 and (time.perf_counter() - t_all) < budget_s:
            t0 = time.perf_counter()
            mod.das(s.Y, s.Gt, s.Gr, s.Ro, np.float32(s.dt), s.delay, np.float32(s.cp), "tfm", "ignore", "cpu", "")
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
            runs += 1
        return {"value": s.sums / best / 1e9, "unit": "Gsum/s", "cores": nproc, "kind": "reference",
                "sample": f"full frame ({s.sums} sums), best of {runs}, reference das_f with "
                          f"DREAM_NUM_THREADS={nproc}"}
    n = 2048
    sel = np.random.default_rng(0).choice(s.Ro.shape[0], n, replace=False)
    t0 = time.perf_counter()
    oracle.das(s.Y, s.Gt, s.Gr, np.asfortranarray(s.Ro[sel]), np.float32(s.dt), s.delay, np.float32(s.cp),
               "tfm", "ignore", np.float32)
    dt = time.perf_counter() - t0
    sums = n * s.Gt.shape[0] * s.Gr.shape[0]
    return {"value": sums / dt / 1e9, "unit": "Gsum/s", "cores": 1, "kind": "port",
            "sample": f"{n} random pixels of the frame ({sums} sums), C restatement, 1 thread"}


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return
    from oracle import oracle
    nproc = os.cpu_count() or 1
    os.environ["DREAM_NUM_THREADS"] = str(nproc)
    s = make_scene(0).astype(np.float32)
    mod = oracle.reference_module("f32")
    kind = "reference" if mod is not None else "port"
    Ro = s.Ro
    sums = s.sums

    def step():
        if mod is not None:
            mod.das(s.Y, s.Gt, s.Gr, Ro, np.float32(s.dt), s.delay, np.float32(s.cp), "tfm", "ignore", "cpu", "")
        else:
            oracle.das(s.Y, s.Gt, s.Gr, Ro, np.float32(s.dt), s.delay, np.float32(s.cp), "tfm", "ignore",
                       np.float32)

    t0 = time.perf_counter()
    step()
    first = time.perf_counter() - t0
    sample = "full frame"
    if first * (args.steps + args.warmup) > 150.0 or mod is None:
        # bound the run: a seeded pixel subset of the frame
        n = max(256, int(Ro.shape[0] * min(1.0, 150.0 / max(first, 1e-3) / (args.steps + args.warmup))))
        if mod is None:
            n = min(n, 2048)
        sel = np.sort(np.random.default_rng(0).choice(s.Ro.shape[0], n, replace=False))
        Ro = np.asfortranarray(s.Ro[sel])
        sums = n * s.Gt.shape[0] * s.Gr.shape[0]
        sample = f"{n} seeded pixels of the frame"
    for _ in range(max(0, args.warmup - 1)):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    val = sums * args.steps / tot / 1e9
    cores = nproc if mod is not None else 1
    line = {"metric": METRIC, "value": val, "unit": "Gsum/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scatterers + noise)",
            "config": {"workload": WORKLOAD, "global_batch": 1, "precision": "das_f (FP32)"},
            "cpu_baseline": {"value": val, "unit": "Gsum/s", "cores": cores, "kind": kind,
                             "sample": f"{sample}, {sums} sums per step, DREAM_NUM_THREADS={nproc}"},
            "e2e": {"value": val, "unit": "Gsum/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def measure_peaks(dev):
    """Project-written microbenchmarks (dream_b200/peaks/peaks.cu): the L2
    gather rates the DAS gathers are bounded by, and the FP32/FP64/integer
    pipe rates, measured on this GPU."""
    import torch
    L = ctypes.CDLL(os.path.join(ROOT, "dream_b200", "libdream_peaks.so"))
    L.dream_peaks_run.restype = ctypes.c_double
    L.dream_peaks_run.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
    log2w = 23  # 32 MiB of floats: L2-resident
    buf = torch.randn(1 << log2w, device=dev)
    blocks, threads = 148 * 8, 256
    sink = torch.zeros(blocks * threads, device=dev)
    ops = ctypes.c_double(0.0)

    def run(kind, iters):
        L.dream_peaks_run(kind, ctypes.c_void_p(buf.data_ptr()), log2w, blocks, threads, 8,
                          ctypes.c_void_p(sink.data_ptr()), ctypes.byref(ops))  # warm-up
        best = None
        for _ in range(3):
            ms = L.dream_peaks_run(kind, ctypes.c_void_p(buf.data_ptr()), log2w, blocks, threads, iters,
                                   ctypes.c_void_p(sink.data_ptr()), ctypes.byref(ops))
            if ms > 0:
                best = ms if best is None else min(best, ms)
        return ops.value / (best * 1e-3) if best else None

    sec = run(0, 512)
    das = run(1, 512)
    f32 = run(2, 4096)
    f64 = run(3, 1024)
    i32 = run(4, 2048)
    return {"l2_random_sector_GBps": sec * 32 / 1e9 if sec else None,
            "l2_random_sector_loads_per_s": sec,
            "l2_das_gather_words_per_s": das, "l2_das_gather_GBps": das * 4 / 1e9 if das else None,
            "fp32_tflops": f32 * 2 / 1e12 if f32 else None, "fp64_tflops": f64 * 2 / 1e12 if f64 else None,
            "int32_tops": i32 / 1e12 if i32 else None,
            "how": "dream_b200/peaks/peaks.cu: 1184 CTAs x 256 threads, best of 3, CUDA events; gathers over "
                   "a 32 MiB L2-resident buffer"}


def read_traffic(kernel_key: str, column: int = 1):
    """Per-launch bytes of a kernel from the committed ncu summary
    (column 1: DRAM read + write, column 2: L2 -> L1 read bytes)."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        parts = line.split()
        if len(parts) > column and parts[0] == kernel_key and not line.startswith("#"):
            try:
                return float(parts[column])
            except ValueError:
                return None
    return None


def l2_roofline(sums: int, step_ms: float, peaks: dict) -> dict:
    """The headline kernel against the measured L2 gather peaks: gathered
    samples per second against the DAS-shaped gather rate, and L2 -> L1 bytes
    (ncu, per launch) per second against the random-sector rate."""
    t = step_ms * 1e-3
    out = {"achieved_words_per_s": sums / t, "gathered_GBps": sums * 4 / t / 1e9,
           "peak_das_gather_words_per_s": peaks.get("l2_das_gather_words_per_s"),
           "peak_l2_random_sector_GBps": peaks.get("l2_random_sector_GBps")}
    out["frac"] = out["achieved_words_per_s"] / out["peak_das_gather_words_per_s"] \
        if out["peak_das_gather_words_per_s"] else None
    l2l1 = read_traffic("das_fast_f32_tfm", 2)
    out["l2_to_l1_bytes_per_launch"] = l2l1
    out["l2_to_l1_GBps"] = l2l1 / t / 1e9 if l2l1 else None
    out["frac_sector"] = out["l2_to_l1_GBps"] / out["peak_l2_random_sector_GBps"] \
        if (l2l1 and out["peak_l2_random_sector_GBps"]) else None
    out["note"] = ("frac: samples/s vs the das-shaped gather microbenchmark; frac_sector: L2->L1 sector "
                   "bytes/s (ncu bytes per launch / live kernel time) vs random 32-byte sector reads")
    return out


def cg_bench(dev, iters: int = 30, reps: int = 3):
    """Model-based reconstruction: 30 CG iterations of (DAS_w DAS_w^T + 1e-3 I)
    x = DAS_w Y on the 32x32 / K=2048 / 256x256 configuration, timed with CUDA
    events on the device (geometry bound once, outside the timing)."""
    import torch
    from dream_b200 import synth
    from dream_b200.autograd import DASOperator, cg_reconstruct
    s = synth.cg_scene(seed=4)
    op = DASOperator(s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", 2048, device=dev)
    xt = torch.from_numpy(s.extra["reflectivity"]).float().to(dev)
    w = torch.ones(op.ncol, device=dev)
    Y = op.adjoint(xt, w)
    cg_reconstruct(op, Y, w, lam=1e-3, iters=2)
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        x, res = cg_reconstruct(op, Y, w, lam=1e-3, iters=iters)
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    # the same solve captured in a CUDA graph (no per-launch host overhead)
    from dream_b200.autograd import CGGraph
    cgg = CGGraph(op, Y, w, lam=1e-3, iters=iters)
    cgg.replay()
    torch.cuda.synchronize()
    ms_graph = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        cgg.replay()
        b.record()
        torch.cuda.synchronize()
        ms_graph.append(a.elapsed_time(b))
    # per-operator timings (gather / scatter) on the same configuration
    def timed(fn, n=10):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / n
    t_g = timed(lambda: op.forward(Y, w))
    t_s = timed(lambda: op.adjoint(xt, w))
    sums = op.No * op.ncol
    corr = float(torch.dot(x, xt) / (x.norm() * xt.norm()))
    return {"config": "TFM 32x32, K=2048, 256x256 image, lam=1e-3, FP32", "iterations": iters,
            "cg_ms": min(ms_graph), "cg_eager_ms": min(ms), "residual_reduction": float(res[-1] / res[0]),
            "corr_with_truth": corr,
            "gather_ms": t_g, "scatter_ms": t_s, "gather_gsum_s": sums / t_g / 1e6,
            "scatter_gsum_s": sums / t_s / 1e6}


def rca_bench(dev, steps: int = 3):
    """The RCA configuration: 128x128 row-column array, row transmit, K=4096,
    128x128x256 grid (68.7e9 sums), A-scans stored in FP32 (268 MB, larger
    than L2) and in BF16; plain FP32 for comparison. Device-resident inputs."""
    import torch
    from dream_b200 import _lib, synth
    from dream_b200.beamformer import grid_hint
    L = _lib.load()
    Y, Gc, Gr_, Ro = synth.rca_frame_torch(device=dev)
    f = lambda a, dt: torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=dt).T)).to(dev).t()
    out = {"config": "RCA 128x128 row-tx, K=4096, 128x128x256 grid", "sums": int(Ro.shape[0]) * 128 * 128}
    d_oob = torch.zeros(1, dtype=torch.int64, device=dev)
    images = {}
    for name, prec in (("plain_f64", _lib.PREC_F64), ("f32_store", _lib.PREC_F32_STORE),
                       ("bf16_store", _lib.PREC_BF16_STORE), ("plain_f32", _lib.PREC_F32)):
        geo = np.float32 if prec == _lib.PREC_F32 else np.float64
        Gt_d, Gr_d, Ro_d, dl = f(Gc, geo), f(Gr_, geo), f(Ro, geo), f(np.zeros((1, 1)), geo)
        if prec == _lib.PREC_BF16_STORE:
            Yd = Y.t().contiguous().to(torch.bfloat16).t()
        elif prec == _lib.PREC_F64:
            Yd = Y.t().contiguous().double().t()
        else:
            Yd = Y
        Im = torch.empty(Ro.shape[0], device=dev, dtype=torch.float64 if prec == _lib.PREC_F64 else torch.float32)
        plan = _lib.plan_create(_lib.RCA_ROWTX, 4096, Ro.shape[0], 128, 128, prec, dev.index)
        _lib.check(L.dream_das_set_grid_hint(plan.handle, grid_hint(Ro)))  # as das / das_f / das_mixed do
        ptr = lambda t: ctypes.c_void_p(t.data_ptr())
        cast = (lambda v: float(np.float32(v))) if prec == _lib.PREC_F32 else float
        args_ = (plan.handle, ptr(Yd), ptr(Ro_d), ptr(Gt_d), ptr(Gr_d), cast(0.025), _lib.DELAY_SINGLE, ptr(dl),
                 cast(1480.0), ptr(Im), ptr(d_oob), ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
        _lib.check(L.dream_das_run_device_async(*args_))
        torch.cuda.synchronize()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            _lib.check(L.dream_das_run_device_async(*args_))
        e.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(e) / steps
        out[name] = {"ms_per_frame": ms, "gsum_s": out["sums"] / ms / 1e6}
        images[name] = Im.double()
        del Yd
    ref = images["plain_f64"]
    scale = float(ref.abs().max())
    for name in ("f32_store", "bf16_store", "plain_f32"):
        out[name]["max_rel_err_vs_fp64"] = float((images[name] - ref).abs().max()) / scale
        out[name]["vs_plain_f64"] = out["plain_f64"]["ms_per_frame"] / out[name]["ms_per_frame"]
    out["error_note"] = ("max |Im - Im_fp64| / max |Im_fp64| over all 4.19M points; Im_fp64 = the plain FP64 kernel "
                         "(bit-identical to the reference das) on the same samples")
    return out


def conv_bench(dev, cpu_sample: bool = True):
    """A-scan synthesis of the reference's TFM test (python/tests/test_das_tfm.py:
    97-105) on the GPU: 101 elements, 2000-sample spatial impulse responses H
    (seeded stand-ins), 150-sample pulse at 50 MHz; per transmit t,
    Hdp = fftconv_p(H, H[:, t]) then Y[:, t*101:(t+1)*101] = conv(Hdp, pulse):
    4.69e10 FP64 multiply-adds, bit-identical to the reference's direct conv().
    Device-resident inputs, CUDA events around all 202 launches."""
    import torch
    from dream_b200.conv import conv_p, fftconv_p
    L, nt, nt_he = 101, 2000, 150
    rng = np.random.default_rng(21)
    H = torch.from_numpy(np.ascontiguousarray(rng.normal(size=(L, nt)))).to(dev).t()  # column-major
    t = np.arange(nt_he) / 50.0
    h_e = torch.from_numpy(-np.exp(-10.0 * (t - 0.55) ** 2) * np.cos(2 * np.pi * 2.5 * t)).to(dev)
    Yfmc = torch.empty((L * L, 2 * nt - 1 + nt_he - 1), dtype=torch.float64, device=dev).t()

    def synth():
        for n_t in range(L):
            Hdp = fftconv_p(H, H[:, n_t])
            conv_p(Hdp, h_e, Yfmc[:, n_t * L:(n_t + 1) * L], "=")

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms = []
        for _ in range(3):
            a.record()
            fn()
            e.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(e))
        return min(ms)

    ms_eager = timed(synth)
    # the same 202 launches captured once in a CUDA graph: device time without
    # the per-call host work of the Python front end
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        synth()
    torch.cuda.current_stream(dev).wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        synth()
    ms = timed(g.replay)
    del g
    # every transmit in two launches (dream_b200.conv.fmc_synthesis), the same A-scans bit for bit
    from dream_b200.conv import fmc_synthesis
    ref_cols = Yfmc[:, 50 * L:51 * L].clone()
    ms_batched = timed(lambda: fmc_synthesis(H, h_e))
    if not torch.equal(fmc_synthesis(H, h_e)[:, 50 * L:51 * L], ref_cols):
        raise RuntimeError("fmc_synthesis differs from the per-transmit fftconv_p calls")
    macs = L * (nt * nt * L + (2 * nt - 1) * nt_he * L)
    out = {"config": "FMC synthesis, 101 elements, SIR 2000 samples, pulse 150 samples, FP64 (reference TFM test)",
           "macs": macs, "ms": ms, "gmac_s": macs / ms / 1e6, "ms_eager": ms_eager,
           "ms_batched": ms_batched, "gmac_s_batched": macs / ms_batched / 1e6,
           "note": "bit-identical to the reference's direct conv(); FFTW's fftconv_p differs by rounding; "
                   "ms: the reference's 202 fftconv_p calls replayed from a CUDA graph, ms_eager: issued from "
                   "Python, ms_batched: all transmits in two launches (fmc_synthesis)"}
    if cpu_sample:
        from concurrent.futures import ThreadPoolExecutor

        from oracle import oracle
        Hh = np.asfortranarray(H.cpu().numpy())
        pulse = h_e.cpu().numpy()
        cores = len(os.sched_getaffinity(0))
        n_tx = min(cores, L)

        def one_transmit(t):  # the oracle's calls release the GIL
            return oracle.conv_p(oracle.conv_p(Hh, Hh[:, t]), pulse)

        t0 = time.perf_counter()
        with ThreadPoolExecutor(n_tx) as ex:
            list(ex.map(one_transmit, range(n_tx)))
        dt_cpu = time.perf_counter() - t0
        out["cpu_port"] = {"gmac_s": n_tx * (macs / L) / dt_cpu / 1e9, "cores": n_tx, "kind": "port",
                           "sample": f"{n_tx} transmits (4.65e8 multiply-adds each), one per host thread, through "
                                     "oracle/conv_oracle.c; the reference's FFTW-based fftconv_p cannot be built "
                                     "here (no FFTW headers)"}
    return out


def arr_example():
    """The reference's array example (examples/rect_arr_example.m): a 21 x 21
    array of 0.9 x 0.9 mm elements at 1 mm pitch (0.03 mm discretisation,
    900 surface elements each), xy focusing at 50 mm, steering -25 degrees in
    x, the field over two 101 x 80 mm planes (x-z and y-z) at 0.5 mm (64722
    points), a 2 mm window at 49-51 mm (dt = 0.1 us, nt = 13, cp = 1500 m/s)."""
    x = np.arange(-10.0, 11.0)
    gx, gy = np.meshgrid(x, x)
    G = np.asfortranarray(np.stack([gx.ravel(order="F"), gy.ravel(order="F"), np.zeros(gx.size)], 1))
    xs, zs = np.arange(-50.0, 50.25, 0.5), np.arange(0.0, 80.25, 0.5)
    X, Z = np.meshgrid(xs, zs)
    xz = np.stack([X.ravel(order="F"), np.zeros(X.size), Z.ravel(order="F")], 1)
    yz = np.stack([np.zeros(X.size), X.ravel(order="F"), Z.ravel(order="F")], 1)
    Ro = np.asfortranarray(np.concatenate([xz, yz]))
    nt = int(round(2.0 * 1e3 / 1500.0 / 0.1))
    n_el = len(np.arange(-0.45 + 0.015, 0.45, 0.03)) ** 2
    return {"Ro": Ro, "G": G, "M": G.shape[0], "geom": [0.9, 0.9], "s_par": [0.03, 0.03, 0.1, nt],
            "delay": (50.0 - 1.0) * 1e3 / 1500.0, "m_par": [1.0, 1500.0, 0.0], "n_el": n_el}


def sir_bench(dev, cpu_sample: bool = True):
    """Spatial impulse responses of a rectangular element (dreamrect, no
    attenuation) on the GPU, bit-identical to the reference: (1) the
    reference's own dreamrect benchmark (python/tests/bench_dreamrect.py: a
    10 x 15 mm element at 0.05 mm = 60000 surface elements, a 61 x 61 x 256
    field of 952576 points, dt = 0.25 us, nt = 300, cp = 1000 m/s: 5.7e10
    surface-element terms, 2.3 GB of SIRs); (2) the reference TFM test's
    element and field line (python/tests/test_das_tfm.py:25-96: 0.4 x 50 mm
    at 0.05 mm, 101 points at z = 10 mm, nt = 2000); (3) dream_arr_rect on
    the reference's array example (arr_example). Device-resident points; the
    unit is one surface-element term."""
    import torch
    from dream_b200.dreamrect import dream_arr_rect, dreamrect
    out = {}

    def timed(fn, n):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(n):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * 1e3 / n

    x = np.linspace(-25.0, 25.0, 101)
    line = np.stack([x, np.zeros_like(x), np.full_like(x, 10.0)], 1)
    X, Yg, Z = np.meshgrid(np.linspace(-15, 15, 61), np.linspace(-15, 15, 61), np.linspace(1.25, 65, 256),
                           indexing="ij")
    field = np.stack([X.ravel(order="F"), Yg.ravel(order="F"), Z.ravel(order="F")], 1)
    cfgs = {"bench_dreamrect": (field, [10.0, 15.0], [0.05, 0.05, 0.25, 300], [1.0, 1000.0, 0.0], 200 * 300, 2),
            "tfm_test_line": (line, [0.4, 50.0], [0.05, 0.05, 0.02, 2000], [1.0, 1500.0, 0.0], 8 * 1000, 3)}
    for name, (Ro, g, sp, mp, n_el, reps) in cfgs.items():
        Rd = torch.from_numpy(np.ascontiguousarray(Ro.T)).to(dev).t()
        ms = timed(lambda: dreamrect(Rd, g, sp, 0.0, mp, "stop"), reps)
        terms = Ro.shape[0] * n_el
        out[name] = {"points": Ro.shape[0], "elements_per_point": n_el, "nt": sp[3], "ms": ms,
                     "gterms_s": terms / ms / 1e6}
        del Rd
        torch.cuda.empty_cache()
    # (3) the reference's array example (examples/rect_arr_example.m)
    arr = arr_example()
    Rd = torch.from_numpy(np.ascontiguousarray(arr["Ro"].T)).to(dev).t()
    ms = timed(lambda: dream_arr_rect(Rd, arr["geom"], arr["G"], arr["s_par"], arr["delay"], arr["m_par"], "xy", 50.0,
                                      "x", [-25.0, 0.0], "off", np.ones(arr["M"]), 1.0, "ignore"), 3)
    terms = arr["Ro"].shape[0] * arr["M"] * arr["n_el"]
    out["rect_arr_example"] = {"points": arr["Ro"].shape[0], "array_elements": arr["M"],
                               "surface_elements": arr["n_el"], "nt": arr["s_par"][3], "ms": ms,
                               "gterms_s": terms / ms / 1e6,
                               "note": "terms the reference evaluates; array elements whose sample window misses "
                                       "[0, nt) for a point are counted out of bounds without being evaluated"}
    del Rd
    torch.cuda.empty_cache()
    if cpu_sample:
        from concurrent.futures import ThreadPoolExecutor

        from oracle import oracle
        cores = len(os.sched_getaffinity(0))

        def threaded(fn, pts):
            # one block of points per host thread (the calls release the GIL)
            blocks = [np.asfortranarray(b) for b in np.array_split(pts, cores) if len(b)]
            t0 = time.perf_counter()
            with ThreadPoolExecutor(cores) as ex:
                res = list(ex.map(fn, blocks))
            return time.perf_counter() - t0, res

        Ro, g, sp, mp, n_el, _ = cfgs["bench_dreamrect"]
        n_s = 16 * cores
        sample = Ro[:: Ro.shape[0] // n_s][:n_s]
        dt_cpu, res = threaded(lambda b: oracle.reference_rect(b, g[0], g[1], sp[0], sp[1], sp[2], sp[3], 0.0, mp[0],
                                                               mp[1]), sample)
        if res and res[0] is not None:
            out["cpu_baseline"] = {"gterms_s": n_s * n_el / dt_cpu / 1e9, "cores": cores, "kind": "reference",
                                   "sample": f"{n_s} points of bench_dreamrect through the reference's "
                                             f"opencl/dreamrect.cl compiled as C (oracle/_ref), {cores} host threads "
                                             "over blocks of points, as the reference's CPU dreamrect threads"}
        n_s = 128 * cores
        sample = arr["Ro"][:: arr["Ro"].shape[0] // n_s][:n_s]
        dt_cpu, _ = threaded(lambda b: oracle.arr_rect(b, arr["geom"][0], arr["geom"][1], arr["G"], arr["s_par"][0],
                                                       arr["s_par"][1], arr["s_par"][2], arr["s_par"][3],
                                                       arr["delay"], 1.0, 1500.0, "xy", 50.0, "x", -25.0, 0.0), sample)
        out["rect_arr_example"]["cpu_baseline"] = {
            "gterms_s": n_s * arr["M"] * arr["n_el"] / dt_cpu / 1e9, "cores": cores, "kind": "port",
            "sample": f"{n_s} points of rect_arr_example through the oracle's dream_arr_rect, {cores} host threads "
                      "over blocks of points (the reference's CPU dream_arr_rect needs FFTW and is not built here)"}
    out["note"] = "wall time around the call (includes the status read-back); unit = one surface-element term"
    return out


def batch_bench(dev, steps: int = 10, n_frames: int = 48):
    """48 uneven TFM frames (elements from {16,32,64,128}, K ~ U{1024..4096},
    cp ~ U[1450,1550], grids 64^2..512^2), FP32, one persistent launch captured
    in a CUDA graph; autotuned tiles. The frames' A-scans (GBs) exceed L2."""
    import torch
    from dream_b200 import synth
    from dream_b200.batch import DASBatch, make_frame
    specs = synth.batch_specs(7, n_frames)
    frames = []
    for sp in specs:
        Y, G, Ro, dt, cp = synth.tfm_frame_torch(sp, device=dev)
        frames.append(make_frame(Y, G, G, Ro, dt, np.zeros((1, 1)), cp, "tfm", device=dev))
        del Y
    t0 = time.perf_counter()
    b = DASBatch(frames)
    tune_s = time.perf_counter() - t0
    g = b.capture()
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        g.replay()
    e.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(e) / steps
    oob_per_batch = b.oob_count() // (steps + 3 + 1)  # the counter accumulates over every replay and the capture run
    return {"config": f"{n_frames} uneven TFM frames, FP32 storage, persistent launch in a CUDA graph",
            "sums_per_batch": b.sums, "in_bounds_sums_per_batch": b.sums - oob_per_batch,
            "oob_sums_per_batch": oob_per_batch, "ms_per_batch": ms, "gsum_s": b.sums / ms / 1e6,
            "in_bounds_gsum_s": (b.sums - oob_per_batch) / ms / 1e6, "work_items": b.items,
            "persistent_ctas": b.grid, "autotune_s": tune_s}


def tfm_extras(dev, scene, plain_f64_ms: float, Im_f64, steps: int = 10, n_copies: int = 8):
    """On the TFM frame itself: the persistent batch kernel over n_copies of
    the frame (the same A-scans, images to separate buffers), and the
    geometry-bound operator's adjoint (scatter) and forward; each against the
    plain FP64 kernel's time on the frame. The batch images are checked
    against the FP64 image (max relative error)."""
    import torch
    from dream_b200.autograd import DASOperator
    from dream_b200.batch import DASBatch, make_frame
    f0 = make_frame(scene.Y, scene.Gt, scene.Gr, scene.Ro, scene.dt, scene.delay, scene.cp, "tfm", device=dev)
    frames = [f0]
    for _ in range(n_copies - 1):
        f = make_frame(f0.Y, f0.Gt, f0.Gr, f0.Ro, scene.dt, scene.delay, scene.cp, "tfm", device=dev)
        frames.append(f)
    b = DASBatch(frames)
    g = b.capture()
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    ms = []
    for i in range(steps):
        flush.fill_(float(i))
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        g.replay()
        e.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(e))
    ms_frame = min(ms) / n_copies
    scale = float(Im_f64.abs().max())
    err = max(float((f.Im.double() - Im_f64).abs().max()) for f in frames) / scale
    out = {"batch_tfm": {"frames": n_copies, "ms_per_frame": ms_frame, "gsum_s": scene.sums / ms_frame / 1e6,
                         "vs_plain_f64": plain_f64_ms / ms_frame, "max_rel_err_vs_fp64": err,
                         "note": "persistent batch kernel over copies of the TFM frame in one CUDA graph; L2 flushed "
                                 "before each replay"}}
    del g, b
    op = DASOperator(scene.Gt, scene.Gr, scene.Ro, scene.dt, scene.delay, scene.cp, "tfm", scene.Y.shape[0],
                     device=dev)
    gen = torch.Generator(device=dev).manual_seed(3)
    x = torch.randn(op.No, device=dev, generator=gen)
    Yd = f0.Y

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        t = []
        for i in range(steps):
            flush.fill_(float(i))
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            e.record()
            torch.cuda.synchronize()
            t.append(a.elapsed_time(e))
        return min(t)
    t_adj = timed(lambda: op.adjoint(x))
    t_fwd = timed(lambda: op.forward(Yd))
    out["adjoint_tfm"] = {"ms_per_frame": t_adj, "gsum_s": scene.sums / t_adj / 1e6,
                          "vs_plain_f64": plain_f64_ms / t_adj,
                          "note": "geometry-bound operator's adjoint (scatter of an N(0,1) image onto the 3000 x 4096 "
                                  "A-scans, zeroing included) on the TFM frame; L2 flushed before each call"}
    out["operator_forward_tfm"] = {"ms_per_frame": t_fwd, "gsum_s": scene.sums / t_fwd / 1e6,
                                   "vs_plain_f64": plain_f64_ms / t_fwd}
    return out


CASES = ("fast_f32", "fast_bf16", "plain_f64", "plain_f32", "saft_fast", "saft_plain_f64", "uni_f32",
         "batch", "op_gather", "op_adjoint", "op_wgrad", "op_backward", "adjoint_tfm", "rca_bf16", "rca_f32",
         "rca_plain_f32", "conv_dp",
         "conv_pulse", "sir_field", "sir_arr", "conv_fmc")


def run_case(name: str, repeat: int = 3):
    """One kernel family on a fixed workload, `repeat` launches after one
    warm-up, for profiling (`ncu -k <kernel> ... bench.py --case NAME`):

      fast_f32 / fast_bf16 / plain_f64 / plain_f32   TFM 64x64, K=3000, 512x512
      saft_fast / saft_plain_f64                     SAFT 64 el, K=2048, 256x256
      uni_f32                                        das_uni TFM 64x64, K=3000, 512x512 (FP32)
      batch                                          the first 12 of the 48 uneven batch frames
      op_gather / op_adjoint / op_wgrad / op_backward  CG configuration 32x32, K=2048, 256x256
      adjoint_tfm                                    the operator's adjoint on the TFM 64x64, K=3000, 512x512 frame
      rca_bf16 / rca_f32                             RCA 128x128 row-tx, K=4096, 128x128x256 grid
      rca_plain_f32                                  the same frame through the plain FP32 kernel (das_f)
      conv_dp / conv_pulse                           fftconv_p of the TFM synthesis: 2000x101 SIRs with a
                                                     2000-sample column / 3999x101 with the 150-sample pulse
      sir_field                                      dreamrect, the reference bench_dreamrect element on a
                                                     16x16x32 subset of its field
      sir_arr                                        dream_arr_rect, the reference's array example (arr_example)
      conv_fmc                                       fmc_synthesis of the TFM test: 101 x 101 double paths of
                                                     2000-sample SIRs, then the 150-sample pulse (two launches)
    Prints one JSON line with the mean wall time per call (not a bench value)."""
    import torch
    from dream_b200 import das, das_f, synth
    from dream_b200.beamformer import das_mixed, das_uni
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    t = lambda a, dt=np.float64: torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=dt).T)).to(dev).t()
    if name in ("fast_f32", "fast_bf16", "plain_f64", "plain_f32", "uni_f32", "adjoint_tfm"):
        sc = synth.tfm_scene(seed=1)
    elif name.startswith("saft"):
        sc = synth.saft_scene(seed=0)
    elif name.startswith("op_"):
        sc = synth.cg_scene(seed=4)
    else:
        sc = None
    if name in ("fast_f32", "fast_bf16"):
        Y = t(sc.Y, np.float32)
        fn = lambda: das_mixed(Y, sc.Gt, sc.Gr, sc.Ro, sc.dt, sc.delay, sc.cp, "tfm", "ignore", "cuda:0",
                               "bf16" if name == "fast_bf16" else "f32", tile=(16, 8))  # the autotuned tile
    elif name in ("plain_f64", "plain_f32", "saft_plain_f64"):
        T = np.float32 if name == "plain_f32" else np.float64
        mod = das_f if T == np.float32 else das
        method = "saft" if name.startswith("saft") else "tfm"
        Y, Gt, Ro, dl = t(sc.Y, T), t(sc.Gt, T), t(sc.Ro, T), t(sc.delay, T)
        Gr = t(sc.Gr, T) if method == "tfm" else None
        fn = lambda: mod.das(Y, Gt, Gr, Ro, T(sc.dt), dl, T(sc.cp), method, "ignore", "cuda:0")
    elif name == "saft_fast":
        Y = t(sc.Y, np.float32)
        fn = lambda: das_mixed(Y, sc.Gt, None, sc.Ro, sc.dt, sc.delay, sc.cp, "saft", "ignore", "cuda:0", "f32")
    elif name == "uni_f32":
        Y = t(sc.Y, np.float32)
        gt = np.array([sc.Gt[0, 0], sc.Gt[1, 0] - sc.Gt[0, 0], sc.Gt[-1, 0]])
        xs, zs = np.unique(sc.Ro[:, 0]), np.unique(sc.Ro[:, 2])
        ro = np.array([[xs[0], xs[1] - xs[0], xs[-1]], [0.0, 1.0, 0.0], [zs[0], zs[1] - zs[0], zs[-1]]])
        fn = lambda: das_uni(Y, gt, gt, ro, np.float32(sc.dt), 0.0, np.float32(sc.cp), "tfm", "ignore", "cuda:0")
    elif name == "batch":
        from dream_b200.batch import DASBatch, make_frame
        frames = []
        for sp in synth.batch_specs(7, 48)[:12]:
            Y, G, Ro, dt, cp = synth.tfm_frame_torch(sp, device=dev)
            frames.append(make_frame(Y, G, G, Ro, dt, np.zeros((1, 1)), cp, "tfm", device=dev))
        b = DASBatch(frames, autotune=False)
        fn = b.run
    elif name.startswith("op_"):
        from dream_b200.autograd import DASOperator
        op = DASOperator(sc.Gt, sc.Gr, sc.Ro, sc.dt, sc.delay, sc.cp, "tfm", 2048, device=dev)
        x = torch.from_numpy(sc.extra["reflectivity"]).float().to(dev)
        w = torch.ones(op.ncol, device=dev)
        Y = op.adjoint(x, w)  # A-scans synthesised from the reflectivity (the CG forward model)
        fn = {"op_gather": lambda: op.forward(Y, w), "op_adjoint": lambda: op.adjoint(x, w),
              "op_wgrad": lambda: op.wgrad(x, Y), "op_backward": lambda: op.backward(x, Y, w)}[name]
    elif name == "adjoint_tfm":
        from dream_b200.autograd import DASOperator
        op = DASOperator(sc.Gt, sc.Gr, sc.Ro, sc.dt, sc.delay, sc.cp, "tfm", sc.Y.shape[0], device=dev)
        x = torch.randn(op.No, device=dev, generator=torch.Generator(device=dev).manual_seed(3))
        fn = lambda: op.adjoint(x)
    elif name == "rca_plain_f32":
        Yr, Gc, Grow, Ro = synth.rca_frame_torch(device=dev)
        f32 = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float32).T)).to(dev).t()
        Gc32, Gr32, Ro32, d32 = f32(Gc), f32(Grow), f32(Ro), f32(np.zeros((1, 1)))
        fn = lambda: das_f.das(Yr, Gc32, Gr32, Ro32, np.float32(0.025), d32, np.float32(1480.0), "rca_rowtx",
                               "ignore", "cuda:0")
    elif name in ("rca_bf16", "rca_f32"):
        Yr, Gc, Grow, Ro = synth.rca_frame_torch(device=dev)
        if name == "rca_bf16":
            Yr = Yr.t().contiguous().to(torch.bfloat16).t()
        fn = lambda: das_mixed(Yr, Gc, Grow, Ro, 0.025, np.zeros((1, 1)), 1480.0, "rca_rowtx", "ignore",
                               "cuda:0", "bf16" if name == "rca_bf16" else "f32")
    elif name in ("conv_dp", "conv_pulse"):
        from dream_b200.conv import fftconv_p
        rng = np.random.default_rng(21)
        M, Lp = (2000, 2000) if name == "conv_dp" else (3999, 150)
        A = torch.from_numpy(np.ascontiguousarray(rng.normal(size=(101, M)))).to(dev).t()
        B = torch.from_numpy(rng.normal(size=Lp)).to(dev)
        fn = lambda: fftconv_p(A, B)
    elif name == "sir_field":
        from dream_b200.dreamrect import dreamrect
        X, Yg, Z = np.meshgrid(np.linspace(-15, 15, 16), np.linspace(-15, 15, 16), np.linspace(1.25, 65, 32),
                               indexing="ij")
        Ro = np.stack([X.ravel(order="F"), Yg.ravel(order="F"), Z.ravel(order="F")], 1)
        Rd = torch.from_numpy(np.ascontiguousarray(Ro.T)).to(dev).t()
        fn = lambda: dreamrect(Rd, [10.0, 15.0], [0.05, 0.05, 0.25, 300], 0.0, [1.0, 1000.0, 0.0], "stop")
    elif name == "conv_fmc":
        from dream_b200.conv import fmc_synthesis
        rng = np.random.default_rng(21)
        Hd = torch.from_numpy(np.ascontiguousarray(rng.normal(size=(101, 2000)))).to(dev).t()
        tp = np.arange(150) / 50.0
        pulse = torch.from_numpy(-np.exp(-10.0 * (tp - 0.55) ** 2) * np.cos(2 * np.pi * 2.5 * tp)).to(dev)
        fn = lambda: fmc_synthesis(Hd, pulse)
    elif name == "sir_arr":
        from dream_b200.dreamrect import dream_arr_rect
        arr = arr_example()
        Rd = torch.from_numpy(np.ascontiguousarray(arr["Ro"].T)).to(dev).t()
        fn = lambda: dream_arr_rect(Rd, arr["geom"], arr["G"], arr["s_par"], arr["delay"], arr["m_par"], "xy", 50.0,
                                    "x", [-25.0, 0.0], "off", np.ones(arr["M"]), 1.0, "ignore")
    else:
        raise SystemExit(f"unknown case {name!r}; one of {', '.join(CASES)}")
    fn()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(repeat):
        fn()
    torch.cuda.synchronize()
    print(json.dumps({"case": name, "launches": repeat, "ms_per_call_wall": (time.perf_counter() - t0) * 1e3 / repeat}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--peaks", action="store_true", help="print the measured roofline peaks and exit")
    ap.add_argument("--case", choices=CASES + ("all",), help="run one kernel family on a fixed workload (profiling)")
    ap.add_argument("--repeat", type=int, default=3, help="calls of --case after one warm-up call")
    args = ap.parse_args()
    if args.case:
        for c in (CASES if args.case == "all" else (args.case,)):
            run_case(c, args.repeat)
        return
    if args.impl == "reference":
        return run_reference(args)
    if args.peaks:
        import torch
        print(json.dumps(measure_peaks(torch.device("cuda", 0))))
        return

    import torch
    import torch.distributed as dist
    from dream_b200 import _lib, das_f

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    L = _lib.load()

    scene = make_scene(rank)
    s32 = scene.astype(np.float32)
    K, C = s32.Y.shape
    No, Nt, Nr = s32.Ro.shape[0], s32.Gt.shape[0], s32.Gr.shape[0]
    sums = s32.sums

    def dev_f(a, dt):  # column-major device copy
        return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=dt).T)).to(dev).t()

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    d_oob = torch.zeros(1, dtype=torch.int64, device=dev)
    from dream_b200.beamformer import grid_hint
    hint = grid_hint(scene.Ro)
    tuned = {}

    def variant(prec_code, steps, warmup):
        geo_dt = np.float32 if prec_code == _lib.PREC_F32 else np.float64
        y_dt = np.float64 if prec_code == _lib.PREC_F64 else np.float32
        Y = dev_f(scene.Y, y_dt)
        if prec_code == _lib.PREC_BF16_STORE:
            Y = Y.t().contiguous().to(torch.bfloat16).t()
        Gt, Gr, Ro = (dev_f(a, geo_dt) for a in (scene.Gt, scene.Gr, scene.Ro))
        delay = dev_f(np.zeros((1, 1)), geo_dt)
        Im = torch.empty(No, dtype=torch.float64 if prec_code == _lib.PREC_F64 else torch.float32, device=dev)
        plan = _lib.plan_create(_lib.TFM, K, No, Nt, Nr, prec_code, local)
        if prec_code in (_lib.PREC_F32_STORE, _lib.PREC_BF16_STORE):
            from dream_b200 import autotune
            cfg = autotune.tune(Y, Gt, Gr, Ro, scene.dt, delay, scene.cp, "tfm",
                                "bf16" if prec_code == _lib.PREC_BF16_STORE else "f32")
            autotune.apply(plan, cfg, Ro)
            tuned[prec_code] = cfg
        ptr = lambda t: ctypes.c_void_p(t.data_ptr())
        cast = (lambda v: float(np.float32(v))) if prec_code == _lib.PREC_F32 else float
        args_ = (plan.handle, ptr(Y), ptr(Ro), ptr(Gt), ptr(Gr), cast(scene.dt), _lib.DELAY_SINGLE,
                 ptr(delay), cast(scene.cp), ptr(Im), ctypes.c_void_p(d_oob.data_ptr()),
                 ctypes.c_void_p(stream.cuda_stream))

        def launch():
            _lib.check(L.dream_das_run_device_async(*args_))

        d_oob.zero_()
        for _ in range(warmup):
            flush.fill_(1.0)
            launch()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        n0 = L.dream_das_plan_launch_count(plan.handle)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.fill_(float(i))  # 256 MiB write evicts the A-scans (49-98 MB) from the 126 MB L2
            evs[i][0].record(stream)
            launch()
            evs[i][1].record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        launches = L.dream_das_plan_launch_count(plan.handle) - n0
        ms = [a.elapsed_time(b) for a, b in evs]
        tot = torch.tensor([sum(ms)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(tot, op=dist.ReduceOp.MAX)
        if int(d_oob.item()) != 0:
            raise RuntimeError("unexpected out-of-bounds terms in the benchmark scene")
        return float(tot.item()), launches, Im

    clocks = ClockSampler(local)
    clocks.start()
    tot_h, launches_h, Im_h = variant(_lib.PREC_F32_STORE, args.steps, args.warmup)
    clk = clocks.stop()
    side = max(3, args.steps // 4)
    others, images = {}, {"f32_store": Im_h.double()}
    for name, code in (("bf16_store", _lib.PREC_BF16_STORE), ("plain_f32", _lib.PREC_F32),
                       ("plain_f64", _lib.PREC_F64)):
        t, _, Im_v = variant(code, side, max(3, args.warmup // 2))
        others[name] = {"gsum_s": world * sums / (t / side * 1e-3) / 1e9, "ms_per_frame": t / side}
        images[name] = Im_v.double()

    step_ms = tot_h / args.steps
    # image error of every variant against the plain FP64 image (bit-identical to the reference das),
    # computed after the timing
    Im64 = images["plain_f64"]
    scale64 = float(Im64.abs().max())
    variants = dict({"f32_store": {"gsum_s": world * sums / (step_ms * 1e-3) / 1e9, "ms_per_frame": step_ms}},
                    **others)
    for name in ("f32_store", "bf16_store", "plain_f32"):
        variants[name]["max_rel_err_vs_fp64"] = float((images[name] - Im64).abs().max()) / scale64
        variants[name]["vs_plain_f64"] = others["plain_f64"]["ms_per_frame"] / variants[name]["ms_per_frame"]
    variants["error_note"] = ("max |Im - Im_fp64| / max |Im_fp64| over all 262,144 points; Im_fp64 = the plain FP64 "
                              "kernel, bit-identical to the reference das (tests/test_gpu_das_parity.py)")
    extras = tfm_extras(dev, scene, others["plain_f64"]["ms_per_frame"], Im64)
    value = world * sums / (step_ms * 1e-3) / 1e9

    # ---- e2e through the public API from pinned host memory ----
    def pinned_f(a, dt):
        a = np.asarray(a, dtype=dt)
        t = torch.empty(a.shape[::-1], dtype=torch.float32 if dt == np.float32 else torch.float64,
                        pin_memory=True)
        arr = t.numpy().T
        arr[...] = a
        return arr

    from dream_b200.beamformer import das_mixed
    hY = pinned_f(scene.Y, np.float32)
    hGt, hGr, hRo = (pinned_f(a, np.float64) for a in (scene.Gt, scene.Gr, scene.Ro))
    hdelay = pinned_f(np.zeros((1, 1)), np.float64)
    e2e_steps = max(10, args.steps)

    def e2e_call():
        return das_mixed(hY, hGt, hGr, hRo, scene.dt, hdelay, scene.cp, "tfm", "ignore", "cuda", "f32")

    # warm up the way the timed loop calls (the previous image alive during the
    # next call), so the pinned host blocks the images land in exist beforehand
    out = None
    for _ in range(max(3, args.warmup)):
        out = e2e_call()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        out = e2e_call()
    t_e2e = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_e2e, op=dist.ReduceOp.MAX)
    e2e_val = world * sums * e2e_steps / float(t_e2e.item()) / 1e9
    h2d = hY.nbytes + hGt.nbytes + hGr.nbytes + hRo.nbytes + hdelay.nbytes
    d2h = out.nbytes + 8

    cg = cg_bench(dev)
    batched = batch_bench(dev)
    rca = rca_bench(dev)
    conv = conv_bench(dev, cpu_sample=(rank == 0 and not args.no_cpu_baseline))
    sir = sir_bench(dev, cpu_sample=(rank == 0 and not args.no_cpu_baseline))
    peaks = measure_peaks(dev)

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return

    hbm_peak, peak_kind = measured_peaks()
    gathered = sums * 4  # one FP32 sample gathered per sum
    achieved = gathered / (step_ms * 1e-3) / 1e9
    compulsory = s32.Y.nbytes + s32.Ro.nbytes + No * 4 + (Nt + Nr) * 12
    l2peak = peaks.get("l2_random_sector_GBps")
    l2l1 = read_traffic("das_fast_f32_tfm", 2)
    line = {
        "metric": METRIC, "value": value, "unit": "Gsum/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded point scatterers, Gaussian-windowed 5 MHz sine, N(0,0.01) noise)",
        "config": {"workload": WORKLOAD, "global_batch": world, "frames_per_gpu": 1,
                   "precision": "FP32-stored A-scans, FP32 compensated sums, FP64-exact sample indices",
                   "l2": "flushed between timed steps (256 MiB write, outside the timed events)",
                   "parallelism": f"{world} independent frames, one per GPU"},
        "variants": variants,
        "batch_tfm": extras["batch_tfm"],
        "adjoint_tfm": extras["adjoint_tfm"],
        "operator_forward_tfm": extras["operator_forward_tfm"],
        "e2e": {"value": e2e_val, "unit": "Gsum/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "api": "dream_b200.beamformer.das_mixed(pinned host arrays, device='cuda', storage='f32')"},
        "roofline": {"bound": "l2", "achieved": achieved, "peak": l2peak, "unit": "GB/s",
                     "frac": achieved / l2peak if l2peak else None,
                     "traffic": read_traffic("das_fast_f32_tfm"),
                     "traffic_source": "profiles/ncu_traffic.txt: dram__bytes_read.sum + dram__bytes_write.sum of "
                                       "one ncu capture of `python bench.py --case fast_f32`",
                     "algorithmic_bytes_per_launch": gathered,
                     "peak_source": "L2 random 32-byte-sector read rate measured in this run (dream_b200/peaks)",
                     "l2_to_l1_bytes_per_launch": l2l1,
                     "l2_sector_frac": (l2l1 / (step_ms * 1e-3) / 1e9 / l2peak) if (l2l1 and l2peak) else None,
                     "hbm_compulsory_frac": compulsory / (step_ms * 1e-3) / 1e9 / hbm_peak,
                     "hbm_peak": hbm_peak, "hbm_peak_source": f"{peak_kind} hbm_gbs",
                     "note": "achieved = gathered sample bytes (4 B per sum) / kernel time, against the rate at "
                             "which L2 serves random sectors; the gathers are served by L1 and L2 (the 49 MB of "
                             "A-scans are L2-resident), so the DRAM traffic is the compulsory bytes only "
                             "(hbm_compulsory_frac). l2_sector_frac = L2->L1 sector bytes per launch (ncu) over "
                             "the kernel time, against the same rate. The kernel is limited by instruction "
                             "issue and gather latency (profiles/das_fast_f32_tfm_64x64_K3000_512x512.md)."},
        "adjoint_cg": cg,
        "batched": batched,
        "rca": rca,
        "conv_fmc": conv,
        "sir_dreamrect": sir,
        "autotuned": {("bf16_store" if k == _lib.PREC_BF16_STORE else "f32_store"): v for k, v in tuned.items()},
        "roofline_l2": l2_roofline(sums, step_ms, peaks),
        "peaks": peaks,
        "gpu_launches": int(launches_h),
        "clocks": clk,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(scene)
    print(json.dumps(line))


if __name__ == "__main__":
    main()
