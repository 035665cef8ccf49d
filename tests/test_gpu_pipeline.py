"""The reference's imaging workflows end to end on the GPU: element SIRs
(dreamrect), A-scan synthesis (fftconv_p: double path, then the pulse),
normalisation and beamforming (das), as python/tests/test_das_tfm.py:19-160,
test_das_saft.py:95-149 and test_das_rca.py:20-183 chain them. At a reduced
size (26 elements at 1 mm pitch, 1000-sample SIRs, the image on a fine grid
around the scatterer) each image equals the same chain through the oracles
bit for bit, and peaks at the scatterer."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

DT = 1 / 50.0        # 50 MHz sampling [us]
NT, NT_HE, CP, Z_PT = 1000, 150, 1500.0, 10.0
SYSTEM_DELAY = 0.55 + 0.21  # the pulse's delay to its maximum [us]


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _workflow(method, rect, conv, das):
    t = np.linspace(0.0, DT * (NT_HE - 1), NT_HE)
    h_e = -np.exp(-10 * (t - 0.55) ** 2) * np.cos(2 * np.pi * 2.5 * t)
    xo = np.linspace(-12.5, 12.5, 26)
    L = xo.shape[0]
    zeros = np.zeros(L)
    line_x = np.asfortranarray(np.stack([xo, zeros, np.full(L, Z_PT)], 1))
    if method == "saft":
        H = rect(line_x, 0.4, 15.0, 0.05, 0.05, DT, NT, 0.0, 1.0, CP)
        Y = conv(conv(H, H), h_e)
    else:
        if method == "tfm":
            Ht = Hr = rect(line_x, 0.4, 50.0, 0.05, 0.05, DT, NT, 0.0, 1.0, CP)
        else:  # rca: columns along x transmit, rows along y receive
            Ht = rect(line_x, 0.4, 50.0, 0.05, 0.05, DT, NT, 0.0, 1.0, CP)
            line_y = np.asfortranarray(np.stack([zeros, xo, np.full(L, Z_PT)], 1))
            Hr = rect(line_y, 50.0, 0.4, 0.05, 0.05, DT, NT, 0.0, 1.0, CP)
        Y = np.zeros((2 * NT - 1 + NT_HE - 1, L * L), order="F")
        for n_t in range(L):
            Y[:, n_t * L:(n_t + 1) * L] = conv(conv(Hr, np.ascontiguousarray(Ht[:, n_t])), h_e)
    Y = np.asfortranarray(Y / np.max(np.abs(Y)))
    Gt = np.asfortranarray(np.stack([xo, zeros, zeros], 1))
    Gr = {"saft": np.zeros((0, 3)), "tfm": Gt, "rca": np.asfortranarray(np.stack([zeros, xo, zeros], 1))}[method]
    X, Z = np.meshgrid(np.linspace(-3.0, 3.0, 25), np.linspace(8.0, 12.0, 33))
    Ro = np.asfortranarray(np.stack([X.ravel(order="F"), np.zeros(X.size), Z.ravel(order="F")], 1))
    Im = das(Y, Gt, Gr, Ro, DT, np.full((1, 1), SYSTEM_DELAY), CP, method)
    return Im, Ro


@pytest.mark.parametrize("method", ["tfm", "saft", "rca"])
def test_workflow_matches_oracle_chain(method):
    from dream_b200 import das as gdas
    from dream_b200.conv import fftconv_p
    from dream_b200.dreamrect import dreamrect
    Im, Ro = _workflow(method,
                       lambda R, a, b, dx, dy, dt, nt, d, v, cp: dreamrect(R, [a, b], [dx, dy, dt, nt], d,
                                                                          [v, cp, 0.0], "stop"),
                       fftconv_p,
                       lambda Y, Gt, Gr, R, dt, d, cp, m: gdas.das(Y, Gt, Gr, R, dt, d, cp, m, "ignore", "cuda"))
    ref, _ = _workflow(method,
                       lambda *a: oracle.rect(*a, err_level="stop")[0],
                       oracle.conv_p,
                       lambda Y, Gt, Gr, R, dt, d, cp, m: oracle.das(Y, Gt, Gr, R, dt, d, cp, m, "ignore",
                                                                     np.float64)[0])
    assert np.array_equal(Im, ref)
    # the scatterer the element-line SIRs describe sits at x = 0, z = 10 mm (SAFT doubles the
    # delay, so the reference's system-delay compensation moves its peak about 0.57 mm up)
    x, z = Ro[np.argmax(np.abs(Im)), [0, 2]]
    assert abs(x) <= 0.5 and abs(z - Z_PT) <= 0.75
