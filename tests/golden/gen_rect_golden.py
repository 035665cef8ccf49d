"""Generates tests/golden/rect_golden.npz by running the reference's
dreamrect kernel (opencl/dreamrect.cl, compiled unmodified as C into
oracle/_ref/libref_dreamrect.so by oracle/build_ref.sh) on rect_cases.py.

    oracle/build_ref.sh && python tests/golden/gen_rect_golden.py

The reference kernel skips out-of-bounds samples silently, i.e. the
err_level 'ignore' behaviour of the CPU dreamrect."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from oracle import oracle  # noqa: E402
from rect_cases import RECT_CASES  # noqa: E402


def main():
    out = {}
    for name, c in RECT_CASES.items():
        H = oracle.reference_rect(c["Ro"], c["a"], c["b"], c["dx"], c["dy"], c["dt"], c["nt"], c["delay"], c["v"],
                                  c["cp"])
        if H is None:
            raise SystemExit("oracle/_ref/libref_dreamrect.so missing: run oracle/build_ref.sh first")
        out[name + "__H"] = H
    np.savez_compressed(os.path.join(HERE, "rect_golden.npz"), **out)
    print("wrote", len(out), "cases")


if __name__ == "__main__":
    main()
