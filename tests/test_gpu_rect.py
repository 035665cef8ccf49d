"""GPU dreamrect (spatial impulse response of a rectangular transducer)
against the reference kernel's stored outputs and the oracle: bit-identical
SIRs through the host and device entries, per-point delays, both SIR
layouts (shared and global memory), error levels."""
import os

import numpy as np
import pytest

from oracle import oracle
from rect_cases import RECT_CASES, random_rect_case

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.fixture(scope="module")
def rect_golden():
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rect_golden.npz"))


def _call(c, err="ignore", delay=None, on_device=False):
    from dream_b200.dreamrect import dreamrect
    d = c["delay"] if delay is None else delay
    Ro = c["Ro"]
    if on_device:
        Ro = torch.from_numpy(np.ascontiguousarray(Ro.T)).cuda().t()
    H = dreamrect(Ro, [c["a"], c["b"]], [c["dx"], c["dy"], c["dt"], c["nt"]], d, [c["v"], c["cp"], 0.0], err)
    return H.cpu().numpy() if on_device else H


@pytest.mark.parametrize("on_device", [False, True])
@pytest.mark.parametrize("name", sorted(RECT_CASES))
def test_matches_reference_kernel(name, on_device, rect_golden):
    H = _call(RECT_CASES[name], on_device=on_device)
    ref = rect_golden[name + "__H"]
    assert H.shape == ref.shape
    assert np.array_equal(H, ref), f"{np.sum(H != ref)} samples differ"


def test_per_point_delay_matches_oracle():
    c = RECT_CASES["square_cloud"]
    d = np.random.default_rng(3).uniform(-0.5, 0.8, (c["Ro"].shape[0], 1))
    ref, _, _ = oracle.rect(c["Ro"], c["a"], c["b"], c["dx"], c["dy"], c["dt"], c["nt"], d, c["v"], c["cp"],
                            "ignore")
    assert np.array_equal(_call(c, delay=d), ref)


@pytest.mark.parametrize("nt", [10000, 30000])  # two warps per CTA in shared memory; global memory
def test_long_responses(nt):
    c = dict(RECT_CASES["neg_delay"], nt=nt, dt=0.0005)
    ref, _, _ = oracle.rect(c["Ro"], c["a"], c["b"], c["dx"], c["dy"], c["dt"], nt, np.full((1, 1), c["delay"]),
                            c["v"], c["cp"], "ignore")
    assert np.array_equal(_call(c), ref)


def test_error_levels(capsys):
    c = RECT_CASES["window_oob"]
    _call(c, "ignore")
    assert "Warning" not in capsys.readouterr().out
    _call(c, "warn")
    assert "Warning: SIR out-of-bounds!" in capsys.readouterr().out
    with pytest.raises(RuntimeError, match="Error in dreamrect"):
        _call(c, "stop")
    H = _call(RECT_CASES["tfm_test_line"], "stop")  # nothing out of bounds: no error
    assert H.shape == (2000, 31)


@pytest.mark.parametrize("seed", range(24))
def test_random_elements_match_oracle(seed):
    c, d = random_rect_case(seed)
    ref, _, _ = oracle.rect(c["Ro"], c["a"], c["b"], c["dx"], c["dy"], c["dt"], c["nt"], d, c["v"], c["cp"], "ignore")
    assert np.array_equal(_call(c, delay=d), ref)


def test_full_size_field_slab_matches_reference():
    """A 61 x 61 x 32 slab (119072 points) of the reference's bench_dreamrect
    field (python/tests/bench_dreamrect.py: 10 x 15 mm element at 0.05 mm,
    nt = 300) against the reference's own CPU dreamrect (oracle/_ref/libref_cpu.so;
    the C restatement when that library is absent), bit for bit."""
    from dream_b200.dreamrect import dreamrect
    X, Yg, Z = np.meshgrid(np.linspace(-15, 15, 61), np.linspace(-15, 15, 61), np.linspace(1.25, 65, 256)[::8],
                           indexing="ij")
    Ro = np.asfortranarray(np.stack([X.ravel(order="F"), Yg.ravel(order="F"), Z.ravel(order="F")], 1))
    args = (Ro, 10.0, 15.0, 0.05, 0.05, 0.25, 300, np.zeros((1, 1)), 1.0, 1000.0)
    ref = oracle.reference_dreamrect(*args, "ignore")
    ref = ref[0] if ref is not None else oracle.rect(*args, "ignore")[0]
    Rd = torch.from_numpy(np.ascontiguousarray(Ro.T)).cuda().t()
    H = dreamrect(Rd, [10.0, 15.0], [0.05, 0.05, 0.25, 300], 0.0, [1.0, 1000.0, 0.0], "stop").cpu().numpy()
    assert bool(np.abs(H).sum() > 0)
    assert np.array_equal(H, ref), f"{np.sum(H != ref)} of {H.size} samples differ"
