"""dreamrect oracle (oracle/rect_oracle.c) pinned against the reference
twice: its OpenCL kernel opencl/dreamrect.cl compiled unmodified as C
(tests/golden/rect_golden.npz, generated by tests/golden/gen_rect_golden.py),
and its CPU dreamrect (src/dreamrect.cc, compiled unmodified into
oracle/_ref/libref_cpu.so; tests/golden/ref_cpu_golden.npz and the live
library on seeded random elements); error levels; the front end's argument
checks (no GPU)."""
import os

import numpy as np
import pytest

from oracle import oracle
from rect_cases import RECT_CASES, random_rect_case


@pytest.fixture(scope="module")
def cpu_golden():
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_cpu_golden.npz"))


@pytest.mark.parametrize("name", sorted(RECT_CASES))
def test_oracle_matches_reference_cpu_dreamrect(name, cpu_golden):
    H, st, oob = _run(RECT_CASES[name])
    assert np.array_equal(H, cpu_golden[f"rect|{name}"])
    assert st == int(cpu_golden[f"rect_st|{name}"])


@pytest.mark.parametrize("seed", range(24))
def test_oracle_matches_live_reference_cpu_dreamrect(seed):
    if oracle.reference_cpu() is None:
        pytest.skip("oracle/_ref/libref_cpu.so not built")
    c, d = random_rect_case(seed)
    args = (c["Ro"], c["a"], c["b"], c["dx"], c["dy"], c["dt"], c["nt"], d, c["v"], c["cp"])
    H, st, _ = oracle.rect(*args, "warn")
    R, st_ref = oracle.reference_dreamrect(*args, "warn")
    assert np.array_equal(H, R) and st == st_ref


@pytest.fixture(scope="module")
def rect_golden():
    import os
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rect_golden.npz"))


def _run(c, err="ignore", delay=None):
    d = np.full((1, 1), c["delay"]) if delay is None else delay
    return oracle.rect(c["Ro"], c["a"], c["b"], c["dx"], c["dy"], c["dt"], c["nt"], d, c["v"], c["cp"], err)


@pytest.mark.parametrize("name", sorted(RECT_CASES))
def test_oracle_matches_reference_kernel(name, rect_golden):
    H, st, oob = _run(RECT_CASES[name])
    assert np.array_equal(H, rect_golden[name + "__H"])


def test_reference_kernel_live_when_built():
    c = RECT_CASES["square_cloud"]
    R = oracle.reference_rect(c["Ro"], c["a"], c["b"], c["dx"], c["dy"], c["dt"], c["nt"], c["delay"], c["v"],
                              c["cp"])
    if R is None:
        pytest.skip("oracle/_ref/libref_dreamrect.so not built")
    assert np.array_equal(_run(c)[0], R)


def test_error_levels():
    c = RECT_CASES["window_oob"]
    _, st_i, oob = _run(c, "ignore")
    _, st_w, _ = _run(c, "warn")
    _, st_s, _ = _run(c, "stop")
    assert oob > 0 and (st_i, st_w, st_s) == (1, 2, 3)
    _, st, oob0 = _run(RECT_CASES["tfm_test_line"], "stop")
    assert st == 0 and oob0 == 0


def test_front_end_argument_errors_without_gpu():
    from dream_b200.dreamrect import dreamrect
    Ro = np.zeros((4, 3))
    with pytest.raises(RuntimeError, match="Error in dreamrect"):
        dreamrect(np.zeros((4, 2)), [1, 1], [0.1, 0.1, 0.02, 100], 0.0, [1, 1500, 0])
    with pytest.raises(RuntimeError, match="Error in dreamrect"):
        dreamrect(Ro, [1, 1, 1], [0.1, 0.1, 0.02, 100], 0.0, [1, 1500, 0])
    with pytest.raises(RuntimeError, match="Error in dreamrect"):
        dreamrect(Ro, [1, 1], [0.1, 0.1, 0.02], 0.0, [1, 1500, 0])
    with pytest.raises(RuntimeError, match="Error in dreamrect"):
        dreamrect(Ro, [1, 1], [0.1, 0.1, 0.02, 100], np.zeros(3), [1, 1500, 0])
    with pytest.raises(RuntimeError, match="attenuation"):
        dreamrect(Ro, [1, 1], [0.1, 0.1, 0.02, 100], 0.0, [1, 1500, 0.5])
