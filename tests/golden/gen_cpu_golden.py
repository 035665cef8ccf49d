"""Generates tests/golden/ref_cpu_golden.npz from the reference's own CPU code
(oracle/_ref/libref_cpu.so, built unmodified by oracle/build_ref.sh with the
FFTW stand-in of oracle/fftw_stub.c; no attenuation):

* conv() (extra_src/conv.cc:33-78) applied column by column as conv_p does, on
  seeded matrices in the three modes '=', '+=' and '-=' (CONV_CASES);
* the CPU dreamrect (src/dreamrect.cc) on every case of rect_cases.py, with
  error level 'ignore' (H and the returned SIRError);
* the CPU dream_arr_rect (src/dream_arr_rect.cc) on every case of
  arr_cases.py, with each case's error level (H and the SIRError).

    oracle/build_ref.sh && python tests/golden/gen_cpu_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from arr_cases import ARR_CASES  # noqa: E402
from oracle import oracle  # noqa: E402
from rect_cases import RECT_CASES  # noqa: E402

# (A rows, A columns, B rows, B columns, seed): B a vector for every column or one column per column
CONV_CASES = {
    "vector_b": (300, 4, 41, 1, 1),
    "matrix_b": (57, 3, 120, 3, 2),
    "short_a": (1, 2, 33, 1, 3),
}


def conv_inputs(name):
    A_M, A_N, B_M, B_N, seed = CONV_CASES[name]
    rng = np.random.default_rng(seed)
    A = np.asfortranarray(rng.normal(size=(A_M, A_N)))
    B = np.asfortranarray(rng.normal(size=(B_M, B_N)))
    Y0 = np.asfortranarray(rng.normal(size=(A_M + B_M - 1, A_N)))
    return A, B, Y0


def arr_args(c):
    return (c["Ro"], c["a"], c["b"], c["G"], c["dx"], c["dy"], c["dt"], c["nt"], c["delay"], c["v"], c["cp"])


def arr_kw(c):
    return dict(foc_met=c["foc_met"], focal=c["focal"], steer_met=c["steer_met"], theta=c["theta"], phi=c["phi"],
                apod_met=c["apod_met"], apod=c["apod"], apod_par=c["apod_par"], err_level=c["err"])


def main():
    if oracle.reference_cpu() is None:
        raise SystemExit("oracle/_ref/libref_cpu.so missing: run oracle/build_ref.sh first")
    out = {}
    for name in CONV_CASES:
        A, B, Y0 = conv_inputs(name)
        for mode in ("=", "+=", "-="):
            out[f"conv|{name}|{mode}"] = oracle.reference_conv_p(A, B, None if mode == "=" else Y0, mode)
    for name, c in RECT_CASES.items():
        H, st = oracle.reference_dreamrect(c["Ro"], c["a"], c["b"], c["dx"], c["dy"], c["dt"], c["nt"],
                                           np.full((1, 1), c["delay"]), c["v"], c["cp"], "ignore")
        out[f"rect|{name}"] = H
        out[f"rect_st|{name}"] = np.array(st)
    for name, c in ARR_CASES.items():
        H, st = oracle.reference_arr_rect(*arr_args(c), **arr_kw(c))
        out[f"arr|{name}"] = H
        out[f"arr_st|{name}"] = np.array(st)
    np.savez_compressed(os.path.join(HERE, "ref_cpu_golden.npz"), **out)
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    main()
