"""GPU dream_arr_rect (spatial impulse responses of arrays of rectangular
elements) against the oracle: bit-identical SIRs through the host and device
entries for every focusing, steering and apodisation method, element
skipping (short windows), shared and global SIR windows, unbounded windows,
warps spanning several elements, out-of-bounds counts and the reference's
status rule; the one-element array against the reference kernel."""
import ctypes
import os

import numpy as np
import pytest

from arr_cases import ARR_CASES, random_case
from gen_arr_golden import ONE_ELEMENT, one_element_points
from oracle import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "arr_golden.npz"))


def _call(c, err=None, on_device=False, G=None, Ro=None):
    from dream_b200.dream_arr_rect import dream_arr_rect
    Ro = c["Ro"] if Ro is None else Ro
    if on_device:
        Ro = torch.from_numpy(np.ascontiguousarray(Ro.T)).cuda().t()
    apod = c["apod"] if c["apod"] is not None else np.ones(c["G"].shape[0])
    H = dream_arr_rect(Ro, [c["a"], c["b"]], c["G"] if G is None else G, [c["dx"], c["dy"], c["dt"], c["nt"]],
                       c["delay"], [c["v"], c["cp"], 0.0], c["foc_met"], c["focal"], c["steer_met"],
                       [c["theta"], c["phi"]], c["apod_met"], apod, 1.0, err or c["err"])
    return H.cpu().numpy() if on_device else H


def _oracle(c, err=None, G=None, Ro=None):
    return oracle.arr_rect(c["Ro"] if Ro is None else Ro, c["a"], c["b"], c["G"] if G is None else G, c["dx"],
                           c["dy"], c["dt"], c["nt"], c["delay"], c["v"], c["cp"], c["foc_met"], c["focal"],
                           c["steer_met"], c["theta"], c["phi"], c["apod_met"], c["apod"], c["apod_par"],
                           err or c["err"])


@pytest.mark.parametrize("on_device", [False, True])
@pytest.mark.parametrize("name", sorted(ARR_CASES))
def test_matches_oracle(name, on_device):
    c = ARR_CASES[name]
    ref, _, _ = _oracle(c, "ignore")
    H = _call(c, "ignore", on_device)
    assert H.shape == ref.shape
    assert np.array_equal(H, ref), f"{np.sum(H != ref)} samples differ"


@pytest.mark.parametrize("name", sorted(ONE_ELEMENT))
def test_one_element_matches_reference_kernel(name, golden):
    from dream_b200.dream_arr_rect import dream_arr_rect
    g, fd, seed, a, b, dx, dy, dt, nt, delay, v, cp = ONE_ELEMENT[name]
    H = dream_arr_rect(one_element_points(seed), [a, b], np.array([g]), [dx, dy, dt, nt], delay, [v, cp, 0.0], "ud",
                       [fd], "off", [0.0, 0.0], "off", [1.0], 1.0, "ignore")
    assert np.array_equal(H, golden[f"one|{name}"])


def test_one_element_at_origin_equals_dreamrect():
    from dream_b200.dreamrect import dreamrect
    c = ARR_CASES["single_origin"]
    R = dreamrect(c["Ro"], [c["a"], c["b"]], [c["dx"], c["dy"], c["dt"], c["nt"]], c["delay"], [c["v"], c["cp"], 0.0],
                  "ignore")
    assert np.array_equal(_call(c, "ignore"), R)


def _counts(c, err):
    """Status and out-of-bounds count through the C ABI."""
    from dream_b200 import _lib
    from dream_b200.dreamrect import APOD_METHODS, FOC_METHODS, STEER_METHODS
    L = _lib.load()
    Ro = np.asfortranarray(c["Ro"])
    G = np.asfortranarray(c["G"])
    d = np.ascontiguousarray(np.asarray(c["delay"], dtype=np.float64).reshape(-1))
    focal = np.ascontiguousarray(np.asarray(c["focal"], dtype=np.float64).reshape(-1))
    apod = None if c["apod"] is None else np.ascontiguousarray(c["apod"], dtype=np.float64)
    H = np.zeros((c["nt"], Ro.shape[0]), order="F")
    oob = ctypes.c_int64(-1)
    p = lambda x: None if x is None else x.ctypes.data_as(ctypes.c_void_p)
    st = L.dream_arr_rect_run(p(Ro), Ro.shape[0], c["a"], c["b"], c["dx"], c["dy"], c["dt"], c["nt"],
                              int(d.size > 1), p(d), c["v"], c["cp"], G.shape[0], p(G), FOC_METHODS[c["foc_met"]],
                              p(focal), STEER_METHODS[c["steer_met"]], c["theta"], c["phi"],
                              APOD_METHODS[c["apod_met"]], p(apod), c["apod_par"], p(H), oracle.ERR_LEVELS[err],
                              ctypes.byref(oob), 0)
    return st, oob.value


@pytest.mark.parametrize("name", ["dead_elements", "example_steered", "ud_3d", "reference_line"])
def test_out_of_bounds_counts_and_status(name):
    c = ARR_CASES[name]
    for err in ("ignore", "warn"):
        _, st_ref, oob_ref = _oracle(c, err)
        st, oob = _counts(c, err)
        assert (st, oob) == (st_ref, oob_ref)
    _, st_ref, oob_ref = _oracle(c, "stop")
    st, _ = _counts(c, "stop")
    assert st == (3 if oob_ref else 0) == st_ref


def test_status_is_the_last_elements():
    c = dict(ARR_CASES["single_origin"], Ro=np.array([[0.0, 0.0, 5.0]]))
    near, far = [0.0, 0.0, 0.0], [0.0, 0.0, -50.0]
    assert _counts(dict(c, G=np.array([far, near])), "warn")[0] == 0
    assert _counts(dict(c, G=np.array([near, far])), "warn")[0] == 2
    with pytest.raises(RuntimeError, match="Error in dream_arr_rect"):
        _call(c, "stop", G=np.array([far, near]))


def test_per_point_delays_and_many_elements():
    # 400 elements of 2 x 3 terms, a delay per point
    c = dict(ARR_CASES["tiny_elements"])
    gx, gy = np.meshgrid(np.linspace(-5, 5, 20), np.linspace(-5, 5, 20))
    c["G"] = np.asfortranarray(np.stack([gx.ravel(), gy.ravel(), np.zeros(400)], 1))
    c["b"], c["dy"] = 0.15, 0.05
    c["delay"] = np.random.default_rng(4).uniform(-0.3, 0.6, c["Ro"].shape[0])
    ref, _, _ = _oracle(c, "ignore")
    assert np.array_equal(_call(c, "ignore"), ref)


def test_empty_shapes():
    c = ARR_CASES["triangle"]
    H = _call(c, "ignore", G=np.zeros((0, 3)))
    assert H.shape == (c["nt"], c["Ro"].shape[0]) and not H.any()
    H = _call(c, "ignore", Ro=np.zeros((0, 3)))
    assert H.shape == (c["nt"], 0)
    H = _call(dict(c, nt=0), "ignore")
    assert H.shape == (0, c["Ro"].shape[0])


def test_host_exception_becomes_a_status():
    # 2^60 elements: the element table's std::vector throws length_error before
    # any allocation (and before the grid is read); the C ABI returns an error
    from dream_b200 import _lib
    L = _lib.load()
    G = np.zeros((1, 3), order="F")
    Ro = np.asfortranarray([[0.0, 0.0, 5.0]])
    d = np.zeros(1)
    H = np.zeros((10, 1), order="F")
    p = lambda x: x.ctypes.data_as(ctypes.c_void_p)
    st = L.dream_arr_rect_run(p(Ro), 1, 1.0, 1.0, 0.1, 0.1, 0.1, 10, 0, p(d), 1.0, 1500.0, 1 << 60, p(G), 0, p(d),
                              0, 0.0, 0.0, 0, None, 0.0, p(H), 1, None, 0)
    assert st == _lib.ERR_ARGUMENT
    assert L.dream_das_last_error()


@pytest.mark.parametrize("seed", range(40))
def test_random_arrays_match_oracle(seed):
    c = random_case(seed)
    ref, st_ref, oob_ref = _oracle(c)
    H = _call(c)
    assert np.array_equal(H, ref, equal_nan=True), f"{np.sum(H != ref)} samples differ"
    assert _counts(c, "warn") == _oracle(c, "warn")[1:]


def test_full_size_array_example_matches_reference():
    """The reference's array example at full size (examples/rect_arr_example.m:
    21 x 21 elements of 0.9 x 0.9 mm, xy focusing at 50 mm, steering -25 deg,
    64722 points on two planes, a 13-sample window) against the reference's own
    CPU dream_arr_rect (oracle/_ref/libref_cpu.so; the C restatement when that
    library is absent), bit for bit, plus the exact scaling in v."""
    from dream_b200.dream_arr_rect import dream_arr_rect
    x = np.arange(-10.0, 11.0)
    gx, gy = np.meshgrid(x, x)
    G = np.asfortranarray(np.stack([gx.ravel(order="F"), gy.ravel(order="F"), np.zeros(gx.size)], 1))
    X, Z = np.meshgrid(np.arange(-50.0, 50.25, 0.5), np.arange(0.0, 80.25, 0.5))
    xz = np.stack([X.ravel(order="F"), np.zeros(X.size), Z.ravel(order="F")], 1)
    Ro = np.asfortranarray(np.concatenate([xz, xz[:, [1, 0, 2]]]))
    delay = 49.0 * 1e3 / 1500.0
    args = (Ro, 0.9, 0.9, G, 0.03, 0.03, 0.1, 13, delay, 1.0, 1500.0)
    kw = dict(foc_met="xy", focal=50.0, steer_met="x", theta=-25.0, phi=0.0, apod_met="off", apod=None,
              apod_par=0.0, err_level="ignore")
    ref = oracle.reference_arr_rect(*args, **kw)
    ref = ref[0] if ref is not None else oracle.arr_rect(*args, **kw)[0]
    Rd = torch.from_numpy(np.ascontiguousarray(Ro.T)).cuda().t()
    run = lambda v: dream_arr_rect(Rd, [0.9, 0.9], G, [0.03, 0.03, 0.1, 13], delay, [v, 1500.0, 0.0], "xy", 50.0,
                                   "x", [-25.0, 0.0], "off", np.ones(G.shape[0]), 1.0, "ignore")
    H1 = run(1.0)
    assert H1.shape == (13, 64722) and bool(H1.abs().sum() > 0)
    H = H1.cpu().numpy()
    assert np.array_equal(H, ref), f"{np.sum(H != ref)} of {H.size} samples differ"
    assert torch.equal(run(2.0), 2 * H1)
