"""The convolution restatement (oracle/conv_oracle.c, direct form of the
reference's conv()) pinned against the reference's own conv()
(extra_src/conv.cc, compiled unmodified into oracle/_ref/libref_cpu.so):
stored outputs in tests/golden/ref_cpu_golden.npz (gen_cpu_golden.py) and the
live library when built; also against numpy.convolve, an independent
implementation, and the front end's argument rules; no GPU."""
import os

import numpy as np
import pytest

from gen_cpu_golden import CONV_CASES, conv_inputs
from oracle import oracle


@pytest.fixture(scope="module")
def cpu_golden():
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_cpu_golden.npz"))


@pytest.mark.parametrize("mode", ["=", "+=", "-="])
@pytest.mark.parametrize("name", sorted(CONV_CASES))
def test_oracle_matches_reference_conv(name, mode, cpu_golden):
    A, B, Y0 = conv_inputs(name)
    Y = oracle.conv_p(A, B, None if mode == "=" else Y0.copy(order="F"), mode)
    assert np.array_equal(Y, cpu_golden[f"conv|{name}|{mode}"])


@pytest.mark.parametrize("seed", range(6))
def test_oracle_matches_live_reference_conv(seed):
    if oracle.reference_cpu() is None:
        pytest.skip("oracle/_ref/libref_cpu.so not built")
    rng = np.random.default_rng(50 + seed)
    A_M, A_N, B_M = (int(v) for v in rng.integers(1, 400, 3))
    A_N = A_N % 6 + 1
    B = rng.normal(size=(B_M, A_N if seed % 2 else 1))
    A = rng.normal(size=(A_M, A_N))
    Y0 = np.asfortranarray(rng.normal(size=(A_M + B_M - 1, A_N)))
    for mode in ("=", "+=", "-="):
        y0 = None if mode == "=" else Y0
        ref = oracle.reference_conv_p(A, B, y0, mode)
        assert np.array_equal(oracle.conv_p(A, B, None if y0 is None else y0.copy(order="F"), mode), ref)


def np_conv(A, B):
    A = np.atleast_2d(A.T).T if A.ndim == 1 else A
    if B.ndim == 1 or 1 in B.shape:
        b = B.reshape(-1)
        return np.stack([np.convolve(A[:, n], b) for n in range(A.shape[1])], 1)
    return np.stack([np.convolve(A[:, n], B[:, n]) for n in range(A.shape[1])], 1)


@pytest.mark.parametrize("shape", [(50, 3, 7, 1), (7, 2, 50, 1), (1, 4, 1, 1), (33, 5, 9, 5), (64, 2, 1, 64)])
def test_oracle_matches_numpy(shape):
    A_M, A_N, B_M, B_N = shape
    rng = np.random.default_rng(sum(shape))
    A = rng.normal(size=(A_M, A_N))
    B = rng.normal(size=(B_M, B_N))
    Y = oracle.conv_p(A, B)
    ref = np_conv(A, B)
    assert Y.shape == ref.shape
    assert np.abs(Y - ref).max() <= 1e-13 * max(np.abs(ref).max(), 1.0)


def test_oracle_in_place_modes():
    rng = np.random.default_rng(2)
    A, B = rng.normal(size=(40, 3)), rng.normal(size=11)
    Y0 = np.asfortranarray(rng.normal(size=(50, 3)))
    add = oracle.conv_p(A, B, Y0.copy(order="F"), "+=")
    sub = oracle.conv_p(A, B, Y0.copy(order="F"), "-=")
    rep = oracle.conv_p(A, B, Y0.copy(order="F"), "=")
    assert np.abs(add - (Y0 + np_conv(A, B))).max() < 1e-13 * np.abs(add).max()
    assert np.abs(sub - (Y0 - np_conv(A, B))).max() < 1e-13 * np.abs(sub).max()
    assert np.array_equal(rep, oracle.conv_p(A, B))


def test_oracle_rejects_mismatched_matrix():
    with pytest.raises(RuntimeError, match="same number of columns"):
        oracle.conv_p(np.ones((5, 3)), np.ones((4, 2)))


def test_front_end_argument_errors_without_gpu():
    from dream_b200.conv import conv_p, fftconv_p
    with pytest.raises(RuntimeError, match="same number of columns as arg 1"):
        fftconv_p(np.ones((5, 3)), np.ones((4, 2)))
    with pytest.raises(RuntimeError, match="Non-valid string in arg 4"):
        conv_p(np.ones((5, 3)), np.ones(4), np.zeros((8, 3), order="F"), "*=")
    with pytest.raises(RuntimeError, match="Wrong number of rows in argument 3"):
        conv_p(np.ones((5, 3)), np.ones(4), np.zeros((7, 3), order="F"), "+=")
    with pytest.raises(RuntimeError, match="Wrong number of columns in argument 3"):
        conv_p(np.ones((5, 3)), np.ones(4), np.zeros((8, 2), order="F"), "+=")
