"""``das`` in FP32: the CUDA counterpart of the reference module ``das_f``
(DAS<float>, python/src/py_das.cc:40-64, built with -DUSE_FLOAT).

    Im = das(Y, Gt, Gr, Ro, dt, delay, cp, method, err_level, device, verbose)
"""
import numpy as np

from .beamformer import das_generic


def das(Y, Gt, Gr, Ro, dt, delay, cp, method, err_level="stop", device="cuda", verbose=""):
    """Delay-and-sum image (1-D, length No) in FP32; see dream_b200.beamformer."""
    return das_generic(np.float32, Y, Gt, Gr, Ro, dt, delay, cp, method, err_level, device, verbose)
