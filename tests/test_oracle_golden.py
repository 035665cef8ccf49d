"""The oracle (C restatement of the reference DAS) against the golden images
produced by the unmodified reference das/das_f (tests/golden/gen_golden.py)."""
import numpy as np
import pytest

from cases import CASES, build_scene, input_digest
from gen_golden import UNI_CASES, materialise_uni, uni_Y
from oracle import oracle


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_das_matches_reference(name, golden):
    g, meta = golden
    spec = CASES[name]
    dtype = np.float64 if spec["prec"] == "f64" else np.float32
    s = build_scene(spec).astype(dtype)
    assert input_digest(s, dtype) == meta[name]["digest"], "synthetic generator drifted"
    Im, st, oob = oracle.das(s.Y, s.Gt, s.Gr, s.Ro, dtype(s.dt), s.delay, dtype(s.cp), s.method,
                             spec["err"], dtype)
    if meta[name]["raised"]:
        assert st == 3 and oob > 0
    else:
        ref = g[name + "__Im"]
        assert Im.dtype == ref.dtype
        assert np.array_equal(Im, ref), f"max diff {np.abs(Im - ref).max()}"
        expect = {"ignore": 1, "warn": 2, "stop": 3}[spec["err"]] if oob else 0
        assert st == expect


@pytest.mark.parametrize("name", sorted(UNI_CASES))
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_oracle_das_uni_matches_reference_das(name, prec, golden):
    g, _ = golden
    method, gt, gr, ro, K, seed = UNI_CASES[name]
    dtype = np.float64 if prec == "f64" else np.float32
    Gt, Gr, Ro = materialise_uni(method, gt, gr, ro, dtype)
    ncols = Gt.shape[0] * (Gr.shape[0] if method != "saft" else 1)
    Y = uni_Y(K, ncols, seed, dtype)
    Im, st, _ = oracle.das_uni(Y, gt, gr, ro, dtype(0.04), 0.0, dtype(1500.0), method, "ignore", dtype)
    assert np.array_equal(Im, g[f"{name}_{prec}__Im"])


def test_index_reveal_is_an_index():
    """With one element pair and Y[:,0] = k+1 the image is the selected index + 1."""
    s = build_scene(CASES["reveal_f64"])
    Im, st, oob, idx = oracle.das(s.Y, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", "ignore",
                                  np.float64, return_idx=True)
    k = idx[0]
    expect = np.where(k == oracle.OOB_MISS, 0, k + 1)
    assert np.array_equal(Im, expect.astype(np.float64))
    assert oob == np.sum(k == oracle.OOB_MISS)


def test_zero_length_ascans_are_all_out_of_bounds():
    Y = np.zeros((0, 4))
    G = np.zeros((2, 3))
    Ro = np.array([[0.0, 0.0, 10.0]])
    Im, st, oob = oracle.das(Y, G, G, Ro, 0.04, 0.0, 1500.0, "tfm", "warn")
    assert st == 2 and oob == 4 and Im[0] == 0.0


def test_adjoint_dot_product_oracle():
    """<A x, y> = <x, A^T y> for the weighted DAS operator on oracle indices."""
    s = build_scene(dict(kind="tfm", kw=dict(seed=3, n_el=6, K=900, nx=12, nz=10)))
    _, _, _, idx = oracle.das(s.Y, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", "ignore",
                              np.float64, return_idx=True)
    rng = np.random.default_rng(0)
    w = rng.normal(size=idx.shape[0])
    Yr = rng.normal(size=(900, idx.shape[0]))
    x = rng.normal(size=idx.shape[1])
    lhs = np.dot(oracle.weighted(idx, Yr, w), x)
    rhs = np.sum(Yr * oracle.adjoint(idx, x, w, 900))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), 1.0)
    # weight gradient of <DAS_w(Y), g> is sum_o g_o Y[k(o,c), c]
    g = x
    dw = oracle.wgrad(idx, g, Yr)
    eps = 1e-6
    for c in (0, 7, 35):
        e = np.zeros_like(w)
        e[c] = eps
        fd = (np.dot(oracle.weighted(idx, Yr, w + e), g) - np.dot(oracle.weighted(idx, Yr, w - e), g)) / (2 * eps)
        assert abs(fd - dw[c]) < 1e-6 * max(1.0, abs(dw[c]))
