"""Randomised parity: random element and image-point geometry, A-scan lengths,
sampling, sound speed, scalar or per-point delays (some terms out of bounds).

* plain FP64 / FP32 kernels: bit-identical to the oracle (image and status);
* FP32-storage kernel: FP64 indices (within 1e-6 of the oracle summing the
  same stored samples) and the oracle's out-of-bounds status.

Hypothesis runs derandomised, so the cases are the same on every run.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
hyp = pytest.importorskip("hypothesis")
from hypothesis import HealthCheck, given, settings  # noqa: E402
from hypothesis import strategies as st  # noqa: E402

from oracle import oracle  # noqa: E402


@st.composite
def problems(draw):
    method = draw(st.sampled_from(["saft", "tfm", "rca_coltx", "rca_rowtx"]))
    rng = np.random.default_rng(draw(st.integers(0, 2**31 - 1)))
    if method.startswith("rca"):
        nc = draw(st.integers(1, 10))
        nr = draw(st.integers(max(1, (2 * nc + 2) // 3), min(3 * nc, 12)))  # edge reads in bounds
        Gt = np.stack([np.sort(rng.uniform(-5, 5, nc)), rng.uniform(-1, 1, nc), rng.uniform(-0.5, 0.5, nc)], 1)
        Gr = np.stack([rng.uniform(-1, 1, nr), np.sort(rng.uniform(-5, 5, nr)), rng.uniform(-0.5, 0.5, nr)], 1)
    else:
        nt = draw(st.integers(1, 12))
        nr = 0 if method == "saft" else draw(st.integers(1, 12))
        Gt = np.stack([rng.uniform(-8, 8, nt), rng.uniform(-2, 2, nt), rng.uniform(-1, 1, nt)], 1)
        Gr = (np.stack([rng.uniform(-8, 8, nr), rng.uniform(-2, 2, nr), rng.uniform(-1, 1, nr)], 1)
              if nr else np.zeros((0, 3)))
    No = draw(st.integers(1, 300))
    Ro = np.stack([rng.uniform(-10, 10, No), rng.uniform(-3, 3, No), rng.uniform(0, 25, No)], 1)
    K = draw(st.integers(1, 900))
    dt = float(rng.uniform(0.01, 0.1))
    cp = float(rng.uniform(1000, 2000))
    if draw(st.booleans()):
        delay = rng.uniform(-0.5, 0.5, (No, 1))
    else:
        delay = np.full((1, 1), float(rng.uniform(-0.5, 0.5)))
    C = Gt.shape[0] * (1 if method == "saft" else Gr.shape[0])
    Y = rng.normal(size=(K, C))
    f = np.asfortranarray
    return method, f(Y), f(Gt), f(Gr), f(Ro), dt, f(delay), cp


SETTINGS = settings(max_examples=60, derandomize=True, deadline=None,
                    suppress_health_check=[HealthCheck.too_slow, HealthCheck.data_too_large])


@SETTINGS
@given(problems())
def test_plain_kernels_bit_exact(prob):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dream_b200 import das, das_f
    method, Y, Gt, Gr, Ro, dt, delay, cp = prob
    for mod, T in ((das, np.float64), (das_f, np.float32)):
        c = lambda a: np.asfortranarray(np.asarray(a, dtype=T))
        ref, st_, oob = oracle.das(c(Y), c(Gt), c(Gr), c(Ro), T(dt), c(delay), T(cp), method, "ignore", T)
        Im = mod.das(c(Y), c(Gt), c(Gr) if method != "saft" else None, c(Ro), T(dt), c(delay), T(cp), method,
                     "ignore", "cuda")
        assert np.array_equal(Im, ref), f"{T.__name__} {method}: {np.sum(Im != ref)} of {Im.size} differ"


@SETTINGS
@given(problems())
def test_fp32_storage_fp64_indices(prob):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dream_b200.beamformer import das_mixed
    method, Y, Gt, Gr, Ro, dt, delay, cp = prob
    Ys = np.asfortranarray(Y.astype(np.float32).astype(np.float64))
    ref, st_, oob = oracle.das(Ys, Gt, Gr, Ro, dt, delay, cp, method, "ignore", np.float64)
    absum, _, _ = oracle.das(np.abs(Ys), Gt, Gr, Ro, dt, delay, cp, method, "ignore", np.float64)
    Im = das_mixed(Y, Gt, Gr if method != "saft" else None, Ro, dt, delay, cp, method, "ignore", "cuda", "f32")
    # FP32 sums of the same samples: error bounded by a few ulp of sum|y|;
    # a wrong index would move a pixel by O(1)
    assert np.all(np.abs(Im - ref) <= 1e-6 * absum + 1e-30)
    if oob:
        with pytest.raises(RuntimeError, match="out-of-bounds"):
            das_mixed(Y, Gt, Gr if method != "saft" else None, Ro, dt, delay, cp, method, "stop", "cuda", "f32")
