"""Runs parity cases on the bounds-checked library (libdream_das_checked.so).

Started by test_gpu_checked.py in a child process with DREAM_DAS_CHECKED=1
(the library choice is fixed when dream_b200 is first imported). Every image
must still match the oracle / golden fixtures, and no gather of any kernel
that ran may have tested an index outside Y. Prints one JSON line.
"""
import json
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests", "golden")):
    sys.path.insert(0, p)

from cases import CASES, build_scene  # noqa: E402
from gen_golden import UNI_CASES, materialise_uni, uni_Y  # noqa: E402

from dream_b200 import _lib, beamformer, das, das_f, synth  # noqa: E402
from oracle import oracle  # noqa: E402

seen = {}


def record():
    for p in getattr(beamformer._tls, "plans", {}).values():
        seen[id(p)] = _lib.check(_lib.load().dream_das_plan_bound_violations(p.handle))


def main():
    L = _lib.load()
    assert _lib.CHECKED and L.dream_das_checked_build() == 1, "not the bounds-checked library"
    g = np.load(os.path.join(ROOT, "tests", "golden", "das_golden.npz"))
    meta = json.loads(bytes(g["__meta__"]).decode())
    mismatches, runs = [], 0
    for name in sorted(CASES):
        if meta[name]["raised"]:
            continue
        spec = CASES[name]
        T = np.float64 if spec["prec"] == "f64" else np.float32
        s = build_scene(spec).astype(T)
        mod = das if spec["prec"] == "f64" else das_f
        Gr = s.Gr if s.method != "saft" else None
        Im = mod.das(s.Y, s.Gt, Gr, s.Ro, T(s.dt), s.delay, T(s.cp), s.method, "ignore", "cuda")
        record()
        runs += 1
        if not np.array_equal(Im, g[name + "__Im"]):
            mismatches.append(name)
        # FP32 / BF16 storage kernels on the same scene
        for storage in ("f32", "bf16"):
            beamformer.das_mixed(s.Y.astype(np.float64), s.Gt, Gr, s.Ro, float(s.dt), s.delay, float(s.cp),
                                 s.method, "ignore", "cuda", storage)
            record()
            runs += 1
    for name in sorted(UNI_CASES):
        method, gt, gr, ro, K, seed = UNI_CASES[name]
        for prec, T in (("f64", np.float64), ("f32", np.float32)):
            Gt, Gr, Ro = materialise_uni(method, gt, gr, ro, T)
            ncols = Gt.shape[0] * (Gr.shape[0] if method != "saft" else 1)
            Im = beamformer.das_uni(uni_Y(K, ncols, seed, T), gt, gr, ro, T(0.04), 0.0, T(1500.0), method)
            record()
            runs += 1
            if not np.array_equal(Im, g[f"{name}_{prec}__Im"]):
                mismatches.append(f"{name}_{prec}")
    # a frame large enough for the tiled fast path with a grid hint, 2-D tiles
    # and full inner chunks (FP64 indices checked against the oracle)
    sc = synth.tfm_scene(n_el=32, K=2000, nx=96, nz=96)
    ref, _, _ = oracle.das(sc.Y, sc.Gt, sc.Gr, sc.Ro, sc.dt, sc.delay, sc.cp, "tfm", "ignore", np.float64)
    Ys = sc.Y.astype(np.float32).astype(np.float64)
    ref32, _, _ = oracle.das(np.asfortranarray(Ys), sc.Gt, sc.Gr, sc.Ro, sc.dt, sc.delay, sc.cp, "tfm",
                             "ignore", np.float64)
    absum, _, _ = oracle.das(np.abs(np.asfortranarray(Ys)), sc.Gt, sc.Gr, sc.Ro, sc.dt, sc.delay, sc.cp,
                             "tfm", "ignore", np.float64)
    Im = beamformer.das_mixed(sc.Y, sc.Gt, sc.Gr, sc.Ro, sc.dt, sc.delay, sc.cp, "tfm", "ignore", "cuda", "f32")
    record()
    runs += 1
    if not np.all(np.abs(Im - ref32) <= 1e-6 * absum + 1e-30):
        mismatches.append("tfm_32el_fast")
    del ref
    torch.cuda.synchronize()
    print(json.dumps({"runs": runs, "plans": len(seen), "violations": int(sum(seen.values())),
                      "mismatches": mismatches}))


if __name__ == "__main__":
    main()
