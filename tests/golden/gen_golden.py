"""Generates tests/golden/das_golden.npz by running the UNMODIFIED reference
``das``/``das_f`` modules (oracle/_ref, built from the reference sources by
oracle/build_ref.sh) on the seeded scenes of cases.py.

Run in a container that has the reference sources:
    oracle/build_ref.sh && python tests/golden/gen_golden.py

Stored per case: the reference image (or the fact that the reference raised,
for err_level 'stop' with out-of-bounds terms), a SHA-256 of the inputs, and
the case spec. das_uni has no reference CPU implementation; its expected
images are the reference ``das`` run on the materialised uniform grids
(see UNI_CASES below), which is exact for delay = 0.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from cases import CASES, build_scene, input_digest  # noqa: E402
from oracle import oracle  # noqa: E402

UNI_CASES = {
    # name: (method, gt, gr, ro 3x3 rows x,y,z / cols min,d,max, K, seed)
    "uni_saft": ("saft", [-3.75, 0.5, 3.75], [], [[-8.0, 0.5, 8.0], [0.0, 1.0, 0.0], [5.0, 0.75, 35.0]],
                 2048, 21),
    "uni_tfm": ("tfm", [-3.75, 0.5, 3.75], [-3.75, 0.5, 3.75],
                [[-8.0, 0.5, 8.0], [0.0, 1.0, 0.0], [5.0, 1.0, 35.0]], 3000, 22),
    "uni_rca_coltx": ("rca_coltx", [-1.5, 0.25, 1.5], [-1.5, 0.25, 1.5],
                      [[-4.0, 1.0, 4.0], [-4.0, 2.0, 4.0], [5.0, 2.5, 20.0]], 2500, 23),
    "uni_rca_rowtx": ("rca_rowtx", [-1.5, 0.25, 1.5], [-1.5, 0.25, 1.5],
                      [[-4.0, 1.0, 4.0], [-4.0, 2.0, 4.0], [5.0, 2.5, 20.0]], 2500, 24),
}


def materialise_uni(method, gt, gr, ro, dtype):
    """Element and pixel arrays equal to what the das_uni kernels generate:
    x = min + n*pitch in the kernel type, y = z = 0 for elements, and pixel
    linear index ny + Ny*(nz + Nz*nx)."""
    T = np.dtype(dtype).type
    cnt = lambda a, d, b: oracle.uni_count(T(a), T(d), T(b), dtype)
    def elems(tri):
        n = cnt(*tri)
        x = np.array([T(tri[0]) + T(i) * T(tri[1]) for i in range(n)], dtype=dtype)
        return np.asfortranarray(np.stack([x, np.zeros(n, dtype), np.zeros(n, dtype)], 1))
    Gt = elems(gt)
    Gr = elems(gr) if len(gr) else np.zeros((0, 3), dtype, order="F")
    if method.startswith("rca"):
        # rows lie along y
        Gr = np.asfortranarray(np.stack([np.zeros(Gr.shape[0], dtype), Gr[:, 0],
                                         np.zeros(Gr.shape[0], dtype)], 1))
    ro = np.asarray(ro, dtype=dtype)
    Nx, Ny, Nz = cnt(*ro[0]), cnt(*ro[1]), cnt(*ro[2])
    pts = []
    for nx in range(Nx):
        for nz in range(Nz):
            for ny in range(Ny):
                pts.append((T(ro[0, 0]) + T(nx) * T(ro[0, 1]), T(ro[1, 0]) + T(ny) * T(ro[1, 1]),
                            T(ro[2, 0]) + T(nz) * T(ro[2, 1])))
    Ro = np.asfortranarray(np.array(pts, dtype=dtype))
    return Gt, Gr, Ro


def uni_Y(K, ncols, seed, dtype):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.normal(0.0, 1.0, (K, ncols)).astype(dtype))


def main():
    os.environ.setdefault("DREAM_NUM_THREADS", str(os.cpu_count() or 1))
    mods = {"f64": oracle.reference_module("f64"), "f32": oracle.reference_module("f32")}
    if mods["f64"] is None or mods["f32"] is None:
        sys.exit("reference modules missing: run oracle/build_ref.sh first")
    out, meta = {}, {}
    for name, spec in CASES.items():
        dtype = np.float64 if spec["prec"] == "f64" else np.float32
        s = build_scene(spec).astype(dtype)
        Gr = s.Gr if s.method != "saft" else np.zeros((0, 3), dtype=dtype, order="F")
        raised = False
        try:
            Im = mods[spec["prec"]].das(s.Y, s.Gt, Gr, s.Ro, dtype(s.dt), s.delay, dtype(s.cp),
                                        s.method, spec["err"], "cpu", "")
            out[name + "__Im"] = np.asarray(Im)
        except RuntimeError:
            raised = True
        meta[name] = dict(spec=spec, raised=raised, digest=input_digest(s, dtype))
        print(f"{name:28s} raised={raised}")
    for name, (method, gt, gr, ro, K, seed) in UNI_CASES.items():
        for prec, dtype in (("f64", np.float64), ("f32", np.float32)):
            Gt, Gr, Ro = materialise_uni(method, gt, gr, ro, dtype)
            ncols = Gt.shape[0] * (Gr.shape[0] if method != "saft" else 1)
            Y = uni_Y(K, ncols, seed, dtype)
            Im = mods[prec].das(Y, Gt, Gr, Ro, dtype(0.04), np.zeros((1, 1), dtype, order="F"),
                                dtype(1500.0), method, "ignore", "cpu", "")
            key = f"{name}_{prec}"
            out[key + "__Im"] = np.asarray(Im)
            meta[key] = dict(uni=[method, gt, gr, ro, K, seed], prec=prec)
            print(f"{key:28s} No={Ro.shape[0]}")
    out["__meta__"] = np.frombuffer(json.dumps(meta, sort_keys=True).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "das_golden.npz"), **out)
    print("wrote", os.path.join(HERE, "das_golden.npz"))


if __name__ == "__main__":
    main()
