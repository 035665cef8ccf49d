"""dream_arr_rect oracle (oracle/rect_oracle.c) pinned against the reference:
the whole element summation against the reference's CPU dream_arr_rect
(src/dream_arr_rect.cc, compiled unmodified into oracle/_ref/libref_cpu.so:
every case of arr_cases.py in tests/golden/ref_cpu_golden.npz, and the live
library on 40 seeded random arrays); per-element focusing / steering /
apodisation against src/arr_functions.cc (compiled unmodified;
tests/golden/arr_golden.npz), one-element arrays against the reference's
dreamrect kernel (opencl/dreamrect.cl), the last-element status rule of
src/dream_arr_rect.cc:209-243, and the front end's argument checks (no GPU)."""
import os

import numpy as np
import pytest

from arr_cases import ARR_CASES, random_case
from gen_cpu_golden import arr_args, arr_kw
from gen_arr_golden import (APOD_PAR, APOD_UD, CP, FOCAL_UD, G7, ONE_ELEMENT, PHI, THETA,
                            one_element_points)
from oracle import oracle


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "arr_golden.npz"))


@pytest.fixture(scope="module")
def cpu_golden():
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_cpu_golden.npz"))


@pytest.mark.parametrize("name", sorted(ARR_CASES))
def test_oracle_matches_reference_cpu_arr_rect(name, cpu_golden):
    c = ARR_CASES[name]
    H, st, oob = oracle.arr_rect(*arr_args(c), **arr_kw(c))
    assert np.array_equal(H, cpu_golden[f"arr|{name}"], equal_nan=True)
    assert st == int(cpu_golden[f"arr_st|{name}"])


@pytest.mark.parametrize("seed", range(40))
def test_oracle_matches_live_reference_cpu_arr_rect(seed):
    if oracle.reference_cpu() is None:
        pytest.skip("oracle/_ref/libref_cpu.so not built")
    c = dict(random_case(seed), err="warn")
    H, st, _ = oracle.arr_rect(*arr_args(c), **arr_kw(c))
    R, st_ref = oracle.reference_arr_rect(*arr_args(c), **arr_kw(c))
    assert np.array_equal(H, R, equal_nan=True)
    # The reference reads the threads' statuses only when it ran more than one
    # thread (src/dream_arr_rect.cc:415-424); a single-threaded run returns
    # SIRError::none whatever its points reported.
    threads = min(os.cpu_count() or 1, c["Ro"].shape[0], int(os.environ.get("DREAM_NUM_THREADS", 1 << 30)))
    assert st == st_ref if threads > 1 else st_ref == 0


COMBOS = [(f, s, a) for f in oracle.FOC_METHODS for s in oracle.STEER_METHODS for a in oracle.APOD_METHODS]


@pytest.mark.parametrize("fm,sm,am", COMBOS)
def test_element_helpers_match_reference(fm, sm, am, golden):
    focal = FOCAL_UD if fm == "ud" else 12.5
    r = oracle.arr_elements(G7, fm, focal, sm, THETA, PHI, am, APOD_UD, APOD_PAR, CP)
    assert np.array_equal(np.stack(r), golden[f"elem|{fm}|{sm}|{am}"])


def test_element_helpers_live_reference_when_built():
    r = oracle.arr_elements(G7, "x+y", 9.0, "xy", 33.0, 21.0, "gauss", None, 1.3, 1540.0, reference=True)
    if r is None:
        pytest.skip("oracle/_ref/libref_arr.so not built")
    assert np.array_equal(np.stack(r), np.stack(oracle.arr_elements(G7, "x+y", 9.0, "xy", 33.0, 21.0, "gauss",
                                                                     None, 1.3, 1540.0)))


@pytest.mark.parametrize("name", sorted(ONE_ELEMENT))
def test_one_element_matches_reference_kernel(name, golden):
    g, fd, seed, a, b, dx, dy, dt, nt, delay, v, cp = ONE_ELEMENT[name]
    H, st, oob = oracle.arr_rect(one_element_points(seed), a, b, np.array([g]), dx, dy, dt, nt, delay, v, cp,
                                 foc_met="ud", focal=[fd])
    assert np.array_equal(H, golden[f"one|{name}"])


def test_single_element_at_origin_is_dreamrect():
    c = ARR_CASES["single_origin"]
    H, st, oob = oracle.arr_rect(c["Ro"], c["a"], c["b"], c["G"], c["dx"], c["dy"], c["dt"], c["nt"], c["delay"],
                                 c["v"], c["cp"])
    R, st_r, oob_r = oracle.rect(c["Ro"], c["a"], c["b"], c["dx"], c["dy"], c["dt"], c["nt"], c["delay"], c["v"],
                                 c["cp"])
    assert np.array_equal(H, R) and (st, oob) == (st_r, oob_r)


def test_elements_sum_close_to_separate_responses():
    # the interleaved sum equals the sum of per-element responses up to rounding
    c = ARR_CASES["x_y_clamped"]
    H, _, _ = oracle.arr_rect(c["Ro"], c["a"], c["b"], c["G"], c["dx"], c["dy"], c["dt"], c["nt"], c["delay"],
                              c["v"], c["cp"], c["foc_met"], c["focal"], c["steer_met"], c["theta"], c["phi"],
                              c["apod_met"], c["apod"])
    foc, steer, w = oracle.arr_elements(c["G"], c["foc_met"], c["focal"], c["steer_met"], c["theta"], c["phi"],
                                        c["apod_met"], c["apod"], 0.0, c["cp"])
    S = np.zeros_like(H)
    for m in range(c["G"].shape[0]):
        Hm, _, _ = oracle.arr_rect(c["Ro"], c["a"], c["b"], c["G"][m:m + 1], c["dx"], c["dy"], c["dt"], c["nt"],
                                   c["delay"], c["v"] * w[m], c["cp"], "ud", [foc[m] + steer[m]])
        S += Hm
    assert np.allclose(H, S, rtol=1e-12, atol=1e-9 * np.abs(H).max())


def _status(c, err, G=None):
    G = c["G"] if G is None else G
    return oracle.arr_rect(c["Ro"], c["a"], c["b"], G, c["dx"], c["dy"], c["dt"], c["nt"], c["delay"], c["v"],
                           c["cp"], err_level=err)


def test_status_is_the_last_elements():
    # two elements: only the first one's terms miss the window
    c = dict(ARR_CASES["single_origin"])
    c["Ro"] = np.array([[0.0, 0.0, 5.0]])
    near, far = [0.0, 0.0, 0.0], [0.0, 0.0, -50.0]  # 'far' lies beyond nt
    _, st_w, oob = _status(c, "warn", np.array([far, near]))
    assert oob > 0 and st_w == 0
    _, st_w, _ = _status(c, "warn", np.array([near, far]))
    _, st_i, _ = _status(c, "ignore", np.array([near, far]))
    assert (st_w, st_i) == (2, 1)
    _, st_s, _ = _status(c, "stop", np.array([far, near]))
    assert st_s == 3


def test_front_end_argument_errors_without_gpu():
    from dream_b200.dream_arr_rect import dream_arr_rect
    Ro, G = np.zeros((4, 3)), np.zeros((3, 3))
    base = dict(Ro=Ro, geom_par=[1, 1], G=G, s_par=[0.1, 0.1, 0.02, 100], delay=0.0, m_par=[1, 1500, 0],
                foc_met="off", focal=0.0, steer_met="off", steer_par=[0, 0], apod_met="off", apod=np.ones(3),
                win_par=1.0)
    bad = [dict(G=np.zeros((3, 2))), dict(foc_met="z"), dict(foc_met="ud", focal=np.zeros(2)),
           dict(foc_met="x", focal=np.zeros(2)), dict(steer_met="diag"), dict(steer_par=[1, 2, 3]),
           dict(apod_met="kaiser"), dict(apod_met="ud", apod=np.ones(2)), dict(Ro=np.zeros((4, 2))),
           dict(s_par=[0.1, 0.1, 0.02])]
    for b in bad:
        with pytest.raises(RuntimeError, match="Error in dream_arr_rect"):
            dream_arr_rect(**{**base, **b})
    with pytest.raises(RuntimeError, match="attenuation"):
        dream_arr_rect(**{**base, "m_par": [1, 1500, 0.5]})
