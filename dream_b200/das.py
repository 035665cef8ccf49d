"""``das`` in FP64: the CUDA counterpart of the reference module ``das``
(DAS<double>, python/src/py_das.cc:66-88).

    Im = das(Y, Gt, Gr, Ro, dt, delay, cp, method, err_level, device, verbose)
"""
import numpy as np

from .beamformer import das_generic


def das(Y, Gt, Gr, Ro, dt, delay, cp, method, err_level="stop", device="cuda", verbose=""):
    """Delay-and-sum image (1-D, length No) in FP64; see dream_b200.beamformer."""
    return das_generic(np.float64, Y, Gt, Gr, Ro, dt, delay, cp, method, err_level, device, verbose)
