"""The reference's TFM workflow (python/tests/test_das_tfm.py:19-160) end to
end on the GPU: element SIRs (dreamrect), full-matrix-capture synthesis
(fftconv_p: double path, then the pulse), normalisation, TFM beamforming (das).
At a reduced size (26 elements at 1 mm pitch, 1000-sample SIRs, the image
on a fine grid around the scatterer) the image equals the same chain through
the oracles bit for bit, and peaks at the scatterer."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _workflow(rect, conv, das):
    Fs = 50.0
    dt = 1 / Fs
    nt, nt_he, cp, z_pt = 1000, 150, 1500.0, 10.0
    t = np.linspace(0.0, dt * (nt_he - 1), nt_he)
    h_e = -np.exp(-10 * (t - 0.55) ** 2) * np.cos(2 * np.pi * 2.5 * t)
    xo = np.linspace(-12.5, 12.5, 26)
    Ro = np.asfortranarray(np.stack([xo, np.zeros_like(xo), np.full_like(xo, z_pt)], 1))
    H = rect(Ro, 0.4, 50.0, 0.05, 0.05, dt, nt, 0.0, 1.0, cp)
    L = xo.shape[0]
    Y = np.zeros((2 * nt - 1 + nt_he - 1, L * L), order="F")
    for n_t in range(L):
        Y[:, n_t * L:(n_t + 1) * L] = conv(conv(H, np.ascontiguousarray(H[:, n_t])), h_e)
    Y = np.asfortranarray(Y / np.max(np.abs(Y)))
    G = np.asfortranarray(np.stack([xo, np.zeros(L), np.zeros(L)], 1))
    X, Z = np.meshgrid(np.linspace(-3.0, 3.0, 25), np.linspace(8.0, 12.0, 33))
    Ro_tfm = np.asfortranarray(np.stack([X.ravel(order="F"), np.zeros(X.size), Z.ravel(order="F")], 1))
    Im = das(Y, G, G, Ro_tfm, dt, np.full((1, 1), 0.55 + 0.21), cp)
    return Im, Ro_tfm


def test_tfm_workflow_matches_oracle_chain():
    from dream_b200 import das as gdas
    from dream_b200.conv import fftconv_p
    from dream_b200.dreamrect import dreamrect
    gpu = _workflow(lambda Ro, a, b, dx, dy, dt, nt, d, v, cp: dreamrect(Ro, [a, b], [dx, dy, dt, nt], d, [v, cp, 0.0],
                                                                          "stop"),
                    fftconv_p,
                    lambda Y, Gt, Gr, Ro, dt, d, cp: gdas.das(Y, Gt, Gr, Ro, dt, d, cp, "tfm", "ignore", "cuda"))
    cpu = _workflow(lambda *a: oracle.rect(*a, err_level="stop")[0],
                    oracle.conv_p,
                    lambda Y, Gt, Gr, Ro, dt, d, cp: oracle.das(Y, Gt, Gr, Ro, dt, d, cp, "tfm", "ignore",
                                                                np.float64)[0])
    Im, Ro_tfm = gpu
    assert np.array_equal(Im, cpu[0])
    # the scatterer the element-line SIRs describe sits at x = 0, z = 10 mm
    x, z = Ro_tfm[np.argmax(np.abs(Im)), [0, 2]]
    assert abs(x) <= 0.5 and abs(z - 10.0) <= 0.5
