"""Golden DAS cases: small seeded scenes whose expected images come from the
unmodified reference ``das``/``das_f`` (built from the reference sources by
oracle/build_ref.sh and run by gen_golden.py in a container that has them).

The inputs are regenerated from seeds at test time (numpy's PCG64 stream is
stable); each case stores a SHA-256 of its inputs so a drifting generator is
caught instead of silently comparing different problems.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from dream_b200 import synth  # noqa: E402


def _index_reveal(K=1500, nx=96, nz=96, delay=0.0, x_rng=(-20.0, 20.0), z_rng=(0.0, 50.0)):
    """One transmitter and one receiver with ``Y[:, 0] = k + 1``, so every pixel
    of the image equals (selected sample index + 1), or 0 when out of bounds."""
    G = np.asfortranarray(np.array([[1.25, 0.0, 0.0]]))
    Y = np.asfortranarray((np.arange(K, dtype=np.float64) + 1.0).reshape(K, 1))
    Ro = synth.grid_xz(nx, nz, x_rng, z_rng)
    return synth.Scene(Y, G, G.copy(order="F"), Ro, 0.04, np.full((1, 1), delay, order="F"),
                       1500.0, "tfm", (nx, nz))


def _near_element(delay):
    """Pixels within 0.1 mm of an element, with a negative delay: products
    ``t_dp * Fs`` fall in (-1, 0), where truncation toward zero selects
    sample 0 (in bounds) rather than -1."""
    G = np.asfortranarray(np.array([[0.0, 0.0, 0.0]]))
    K = 64
    Y = np.asfortranarray((np.arange(K, dtype=np.float64) + 1.0).reshape(K, 1))
    Ro = synth.grid_xz(9, 8, (-0.1, 0.1), (0.0, 0.05))
    return synth.Scene(Y, G, G.copy(order="F"), Ro, 0.04, np.full((1, 1), delay, order="F"),
                       1500.0, "tfm", (9, 8))


def _delay_vector(scene, seed):
    rng = np.random.default_rng(seed)
    No = scene.Ro.shape[0]
    scene.delay = np.asfortranarray(rng.uniform(0.0, 0.6, (No, 1)))
    return scene


def build_scene(spec: dict) -> synth.Scene:
    kind = spec["kind"]
    kw = dict(spec.get("kw", {}))
    if kind == "saft":
        s = synth.saft_scene(**kw)
    elif kind == "tfm":
        s = synth.tfm_scene(**kw)
    elif kind == "rca":
        s = synth.rca_scene(**kw)
    elif kind == "index_reveal":
        s = _index_reveal(**kw)
    elif kind == "near_element":
        s = _near_element(**kw)
    else:
        raise ValueError(kind)
    if "delay" in spec:
        s.delay = np.full((1, 1), float(spec["delay"]), order="F")
    if spec.get("delay_vector_seed") is not None:
        s = _delay_vector(s, spec["delay_vector_seed"])
    if "method" in spec:
        s.method = spec["method"]
    return s


def input_digest(s: synth.Scene, dtype) -> str:
    h = hashlib.sha256()
    for a in (s.Y, s.Gt, s.Gr, s.Ro, s.delay):
        h.update(np.ascontiguousarray(np.asarray(a, dtype=dtype)).tobytes())
    h.update(np.asarray([s.dt, s.cp], dtype=dtype).tobytes())
    h.update(s.method.encode())
    return h.hexdigest()


# name -> spec. "prec" is the reference module: f64 -> das, f32 -> das_f.
CASES = {}
for prec in ("f64", "f32"):
    CASES[f"saft_{prec}"] = dict(kind="saft", kw=dict(seed=10, n_el=16, K=2048, nx=24, nz=32),
                                 prec=prec, err="ignore")
    CASES[f"tfm_{prec}"] = dict(kind="tfm", kw=dict(seed=11, n_el=16, K=3000, nx=32, nz=32),
                                prec=prec, err="stop")
    CASES[f"tfm_delay_{prec}"] = dict(kind="tfm", kw=dict(seed=11, n_el=16, K=3000, nx=32, nz=32),
                                      delay=0.37, prec=prec, err="stop")
    CASES[f"tfm_delayvec_{prec}"] = dict(kind="tfm", kw=dict(seed=13, n_el=8, K=3000, nx=16, nz=40),
                                         delay_vector_seed=5, prec=prec, err="ignore")
    CASES[f"rca_coltx_{prec}"] = dict(kind="rca", kw=dict(seed=12, n_cols=12, n_rows=12, K=4096, nx=6,
                                                          ny=6, nz=8, method="rca_coltx"),
                                      prec=prec, err="stop", delay=0.11)
    CASES[f"rca_rowtx_{prec}"] = dict(kind="rca", kw=dict(seed=12, n_cols=12, n_rows=12, K=4096, nx=6,
                                                          ny=6, nz=8, method="rca_rowtx"),
                                      prec=prec, err="stop", delay=0.11)
    CASES[f"rca_alias_{prec}"] = dict(kind="rca", kw=dict(seed=14, n_cols=12, n_rows=12, K=4096, nx=4,
                                                          ny=5, nz=6, method="rca_coltx"),
                                      method="rca", prec=prec, err="ignore")
    # num_cols != num_rows: the stripe edges are read with the reference's
    # literal (mixed) indexing.
    CASES[f"rca_mixed_coltx_{prec}"] = dict(kind="rca", kw=dict(seed=15, n_cols=8, n_rows=10, K=4096, nx=5,
                                                                ny=7, nz=6, method="rca_coltx"),
                                            prec=prec, err="ignore")
    CASES[f"rca_mixed_rowtx_{prec}"] = dict(kind="rca", kw=dict(seed=15, n_cols=8, n_rows=10, K=4096, nx=5,
                                                                ny=7, nz=6, method="rca_rowtx"),
                                            prec=prec, err="ignore")
    # Short A-scans: many terms fall outside [0, K).
    for lvl in ("ignore", "warn", "stop"):
        CASES[f"tfm_oob_{lvl}_{prec}"] = dict(kind="tfm", kw=dict(seed=16, n_el=8, K=700, nx=16, nz=16),
                                              prec=prec, err=lvl)
    CASES[f"saft_oob_{prec}"] = dict(kind="saft", kw=dict(seed=17, n_el=8, K=400, nx=16, nz=16),
                                     prec=prec, err="warn")
    CASES[f"reveal_{prec}"] = dict(kind="index_reveal", kw=dict(), prec=prec, err="ignore")
    CASES[f"reveal_delay_{prec}"] = dict(kind="index_reveal", kw=dict(delay=1.3), prec=prec, err="ignore")
    CASES[f"near_element_{prec}"] = dict(kind="near_element", kw=dict(delay=-0.03), prec=prec, err="ignore")
    CASES[f"near_element_oob_{prec}"] = dict(kind="near_element", kw=dict(delay=-0.045), prec=prec,
                                             err="warn")


RCA_SLABS = (0, 101, 255)  # z-planes of the RCA configuration's 128 x 128 x 256 grid (z is the fastest index)


def rca_slab_points(nz=256, n_xy=128 * 128, slabs=RCA_SLABS):
    """Indices of every (x, y) point of the given z-planes of synth.grid_xyz."""
    return np.sort(np.concatenate([iz + nz * np.arange(n_xy) for iz in slabs]))
