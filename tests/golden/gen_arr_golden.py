"""Generates tests/golden/arr_golden.npz from the reference itself:

* the per-element focusing delays, steering delays and weights of
  src/arr_functions.cc (compiled unmodified with oracle/ref_arr_driver.cc
  into oracle/_ref/libref_arr.so) for every focusing x steering x
  apodisation method on a seeded 7-element array, and
* one-element arrays (an element off the origin, a focusing delay) through
  the reference's dreamrect kernel (opencl/dreamrect.cl, compiled as C into
  oracle/_ref/libref_dreamrect.so), observation points shifted by the element
  centre and the delay reduced by the element's delay, as
  src/dream_arr_rect.cc:227-234 passes them on.

    oracle/build_ref.sh && python tests/golden/gen_arr_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402

# the array and settings of the element-helper fixtures
G7 = np.asfortranarray(np.stack([np.linspace(-3, 5, 7), np.linspace(-1, 2, 7) ** 2, np.linspace(0, 0.3, 7)], 1))
FOCAL_UD = np.linspace(0.1, 1.0, 7)
APOD_UD = np.linspace(0.3, 1.2, 7)
THETA, PHI, APOD_PAR, CP = 17.0, -9.0, 0.7, 1480.0

# one-element cases: (element centre, focusing delay via 'ud', Ro seed, a, b, dx, dy, dt, nt, delay, v, cp)
ONE_ELEMENT = {
    "offset_x": ((1.5, 0.0, 0.0), 0.37, 21, 1.0, 2.0, 0.05, 0.05, 0.02, 700, 0.1, 1.0, 1500.0),
    "offset_xyz": ((-0.8, 1.1, 0.4), -0.25, 22, 0.6, 0.9, 0.03, 0.03, 0.01, 1500, 0.0, 2.0, 1540.0),
}


def one_element_points(seed):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(np.stack([rng.uniform(-3, 3, 10), rng.uniform(-3, 3, 10), rng.uniform(2, 9, 10)], 1))


def main():
    out = {}
    for fm in oracle.FOC_METHODS:
        for sm in oracle.STEER_METHODS:
            for am in oracle.APOD_METHODS:
                focal = FOCAL_UD if fm == "ud" else 12.5
                r = oracle.arr_elements(G7, fm, focal, sm, THETA, PHI, am, APOD_UD, APOD_PAR, CP, reference=True)
                if r is None:
                    raise SystemExit("oracle/_ref/libref_arr.so missing: run oracle/build_ref.sh first")
                out[f"elem|{fm}|{sm}|{am}"] = np.stack(r)
    for name, (g, fd, seed, a, b, dx, dy, dt, nt, delay, v, cp) in ONE_ELEMENT.items():
        Ro = one_element_points(seed)
        shifted = np.asfortranarray(Ro - np.asarray(g)[None, :])
        H = oracle.reference_rect(shifted, a, b, dx, dy, dt, nt, (delay - fd) - 0.0, v, cp)
        if H is None:
            raise SystemExit("oracle/_ref/libref_dreamrect.so missing: run oracle/build_ref.sh first")
        out[f"one|{name}"] = H
    np.savez_compressed(os.path.join(HERE, "arr_golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
