"""GPU column-wise convolution (conv_p / fftconv_p) against the restatement
of the reference's direct conv(): bit-identical images of every shape and
mode, through the host entry (NumPy) and the device entry (CUDA tensors);
within 1e-12 of numpy.convolve, as FFTW's fftconv_p would be."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


SHAPES = [  # A_M, A_N, B_M, B_N
    (2000, 7, 150, 1),      # SIR x pulse (the reference TFM test's second step)
    (2000, 5, 2000, 1),     # SIR x SIR (its double-path step)
    (3999, 3, 150, 1),
    (1, 3, 1, 1),
    (5, 2, 300, 1),         # pulse longer than the signal
    (300, 4, 17, 4),        # one pulse per column
    (1000, 2, 9000, 1),     # pulse beyond the shared-memory budget: global-memory kernel
    (2049, 3, 1, 3),
    (4096, 2, 2047, 1),     # several CTA tiles, ragged last tile
]


def _inputs(shape, seed=0):
    A_M, A_N, B_M, B_N = shape
    rng = np.random.default_rng(seed + A_M + 7 * B_M)
    A = np.asfortranarray(rng.normal(size=(A_M, A_N)))
    B = np.asfortranarray(rng.normal(size=(B_M, B_N)))
    return A, B


@pytest.mark.parametrize("shape", SHAPES)
def test_fftconv_p_bit_exact(shape):
    from dream_b200.conv import fftconv_p
    A, B = _inputs(shape)
    Y = fftconv_p(A, B)
    ref = oracle.conv_p(A, B)
    assert Y.shape == ref.shape and Y.flags["F_CONTIGUOUS"]
    assert np.array_equal(Y, ref)
    vec = B.shape[0] == 1 or B.shape[1] == 1  # a vector in either orientation (the reference's rule)
    npref = np.stack([np.convolve(A[:, n], B.reshape(-1) if vec else B[:, n]) for n in range(A.shape[1])], 1)
    assert np.abs(Y - npref).max() <= 1e-12 * np.abs(npref).max()


@pytest.mark.parametrize("mode", ["=", "+=", "-="])
@pytest.mark.parametrize("shape", [(2000, 3, 150, 1), (300, 4, 17, 4), (1000, 2, 9000, 1)])
def test_conv_p_in_place_modes_bit_exact(shape, mode):
    """In-place modes, starting from values that include -0 and exact zeros
    next to the column ends (where the kernels' padded terms must leave a
    stored -0 untouched, as the reference never visits them)."""
    from dream_b200.conv import conv_p
    A, B = _inputs(shape, 1)
    rng = np.random.default_rng(5)
    Y0 = np.asfortranarray(rng.normal(size=(A.shape[0] + B.shape[0] - 1, A.shape[1])))
    Y0[:3, :] = -0.0
    Y0[-3:, :] = -0.0
    A[:2, :] = 0.0
    A[-2:, :] = 0.0
    ref = oracle.conv_p(A, B, Y0.copy(order="F"), mode)
    Y = Y0.copy(order="F")
    out = conv_p(A, B, Y, mode)
    assert out is Y
    assert np.array_equal(np.signbit(Y), np.signbit(ref)) and np.array_equal(Y, ref)


@pytest.mark.parametrize("shape", [(2000, 5, 150, 1), (300, 4, 17, 4)])
def test_device_tensors(shape):
    """CUDA tensors stay on the device; the same bits as the host entry."""
    from dream_b200.conv import conv_p, fftconv_p
    A, B = _inputs(shape, 2)
    At = torch.from_numpy(A).cuda()
    Bt = torch.from_numpy(B).cuda()
    Yt = fftconv_p(At, Bt)
    assert Yt.is_cuda and Yt.dtype == torch.float64
    ref = oracle.conv_p(A, B)
    assert np.array_equal(Yt.cpu().numpy(), ref)
    Y0 = np.asfortranarray(np.random.default_rng(3).normal(size=ref.shape))
    Yd = torch.from_numpy(np.ascontiguousarray(Y0.T)).cuda().t()
    conv_p(At, Bt, Yd, "+=")
    assert np.array_equal(Yd.cpu().numpy(), oracle.conv_p(A, B, Y0.copy(order="F"), "+="))


def test_empty_signal_and_row_vector_pulse():
    from dream_b200.conv import fftconv_p
    Y = fftconv_p(np.zeros((0, 3)), np.ones(4))
    assert Y.shape == (3, 3) and np.all(Y == 0.0)
    A, B = _inputs((64, 3, 10, 1))
    assert np.array_equal(fftconv_p(A, B.reshape(1, -1)), oracle.conv_p(A, B))


def test_reference_tfm_synthesis_columns():
    """The two convolution steps of the reference's TFM test
    (python/tests/test_das_tfm.py:97-105) for one transmit: SIRs (2000 x 101)
    with the transmit column, then with the 150-sample pulse."""
    from dream_b200.conv import fftconv_p
    rng = np.random.default_rng(11)
    H = np.asfortranarray(rng.normal(size=(2000, 101)))
    t = np.arange(150) / 50.0
    h_e = -np.exp(-10.0 * (t - 0.55) ** 2) * np.cos(2 * np.pi * 2.5 * t)
    Hdp = fftconv_p(H, H[:, 7])
    assert np.array_equal(Hdp, oracle.conv_p(H, H[:, 7]))
    Y = fftconv_p(Hdp, h_e)
    assert Y.shape == (4148, 101)
    assert np.array_equal(Y, oracle.conv_p(Hdp, h_e))


@pytest.mark.parametrize("receive", ["same", "other"])
def test_fmc_synthesis_equals_per_transmit_calls(receive):
    # the reference tests' loop: two fftconv_p calls per transmit (TFM: Hr = Ht; RCA: separate receive SIRs)
    from dream_b200.conv import fftconv_p, fmc_synthesis
    rng = np.random.default_rng(8)
    Ht = np.asfortranarray(rng.normal(size=(300, 7)))
    Hr = Ht if receive == "same" else np.asfortranarray(rng.normal(size=(300, 5)))
    pulse = rng.normal(size=40)
    Y = fmc_synthesis(torch.from_numpy(np.ascontiguousarray(Ht.T)).cuda().t(), pulse,
                      None if receive == "same" else torch.from_numpy(np.ascontiguousarray(Hr.T)).cuda().t())
    L_r = Hr.shape[1]
    assert tuple(Y.shape) == (2 * 300 - 1 + 40 - 1, 7 * L_r)
    Yh = Y.cpu().numpy()
    for t in range(7):
        loop = fftconv_p(fftconv_p(Hr, Ht[:, t]), pulse)
        assert np.array_equal(Yh[:, t * L_r:(t + 1) * L_r], loop)
    assert np.array_equal(Yh[:, 3 * L_r:4 * L_r], oracle.conv_p(oracle.conv_p(Hr, Ht[:, 3]), pulse))
    # host arrays in, host array out
    assert np.array_equal(fmc_synthesis(Ht, pulse, None if receive == "same" else Hr), Yh)
