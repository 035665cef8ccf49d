"""Parity of the plain CUDA kernels (das FP64 / das_f FP32 / das_uni) with the
reference, through the C ABI.

Bar: bit-exact. The plain kernels select the same sample index for every term
and sum each pixel's terms in the reference order, so images must equal the
reference's exactly (np.array_equal), not merely within 1e-12 / 1e-5.
"""
import numpy as np
import pytest

from cases import rca_slab_points, CASES, build_scene
from gen_golden import UNI_CASES, materialise_uni, uni_Y
from oracle import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _mod(prec):
    from dream_b200 import das, das_f
    return das if prec == "f64" else das_f


def _run(prec, s, err, via):
    dtype = np.float64 if prec == "f64" else np.float32
    mod = _mod(prec)
    Gr = s.Gr if s.method != "saft" else None
    if via == "host":
        return mod.das(s.Y, s.Gt, Gr, s.Ro, dtype(s.dt), s.delay, dtype(s.cp), s.method, err, "cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda() if a is not None else None
    out = mod.das(t(s.Y), t(s.Gt), t(Gr), t(s.Ro), dtype(s.dt), t(s.delay), dtype(s.cp), s.method, err,
                  "cuda")
    return out.cpu().numpy()


@pytest.mark.parametrize("via", ["host", "device"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_bit_exact(name, via, golden, capsys):
    g, meta = golden
    spec = CASES[name]
    dtype = np.float64 if spec["prec"] == "f64" else np.float32
    s = build_scene(spec).astype(dtype)
    if meta[name]["raised"]:
        with pytest.raises(RuntimeError, match="out-of-bounds"):
            _run(spec["prec"], s, spec["err"], via)
        return
    Im = _run(spec["prec"], s, spec["err"], via)
    ref = g[name + "__Im"]
    assert Im.dtype == ref.dtype and Im.shape == ref.shape
    assert np.array_equal(Im, ref), f"{np.sum(Im != ref)} pixels differ, max {np.abs(Im - ref).max()}"
    _, st, oob = oracle.das(s.Y, s.Gt, s.Gr, s.Ro, dtype(s.dt), s.delay, dtype(s.cp), s.method,
                            spec["err"], dtype)
    out = capsys.readouterr().out
    assert ("Warning: DAS out-of-bounds!" in out) == (st == 2)


@pytest.mark.parametrize("name", sorted(UNI_CASES))
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("via", ["host", "device"])
def test_das_uni_bit_exact(name, prec, via, golden):
    from dream_b200.beamformer import das_uni
    g, _ = golden
    method, gt, gr, ro, K, seed = UNI_CASES[name]
    dtype = np.float64 if prec == "f64" else np.float32
    Gt, Gr, Ro = materialise_uni(method, gt, gr, ro, dtype)
    ncols = Gt.shape[0] * (Gr.shape[0] if method != "saft" else 1)
    Y = uni_Y(K, ncols, seed, dtype)
    if via == "device":
        Y = torch.from_numpy(np.ascontiguousarray(Y)).cuda()
    Im = das_uni(Y, gt, gr, ro, dtype(0.04), 0.0, dtype(1500.0), method)
    Im = Im.cpu().numpy() if via == "device" else Im
    assert np.array_equal(Im, g[f"{name}_{prec}__Im"])


@pytest.mark.parametrize("method", ["saft", "tfm", "rca_coltx", "rca_rowtx"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_das_uni_with_delay_matches_oracle(method, prec):
    """Non-zero delay: das_uni row-tx adds it to the row leg; the oracle restates that."""
    from dream_b200.beamformer import das_uni
    dtype = np.float64 if prec == "f64" else np.float32
    gt, gr = [-2.0, 0.25, 2.0], ([] if method == "saft" else [-2.0, 0.25, 2.0])
    ro = [[-5.0, 0.5, 5.0], [-3.0, 1.5, 3.0], [4.0, 0.7, 24.0]]
    n = oracle.uni_count(*np.asarray(gt, dtype), dtype)
    ncols = n if method == "saft" else n * n
    Y = uni_Y(2500, ncols, 9, dtype)
    ref, st, oob = oracle.das_uni(Y, gt, gr, ro, dtype(0.04), 0.33, dtype(1500.0), method, "ignore", dtype)
    Im = das_uni(Y, gt, gr, ro, dtype(0.04), 0.33, dtype(1500.0), method)
    assert np.array_equal(Im, ref)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_index_reveal_full_grid(prec):
    """512x512 grid of the TFM configuration, one element pair, Y[:,0] = k+1:
    every pixel's value is its selected sample index + 1 (0 when out of bounds)."""
    from cases import _index_reveal
    dtype = np.float64 if prec == "f64" else np.float32
    s = _index_reveal(K=3000, nx=512, nz=512, x_rng=(-20.0, 20.0), z_rng=(2.0, 50.0)).astype(dtype)
    ref, st, oob, idx = oracle.das(s.Y, s.Gt, s.Gr, s.Ro, dtype(s.dt), s.delay, dtype(s.cp), "tfm",
                                   "ignore", dtype, return_idx=True)
    Im = _run(prec, s, "ignore", "device")
    assert np.array_equal(Im, ref)
    k = np.where(idx[0] == oracle.OOB_MISS, -1, idx[0])
    assert np.array_equal(Im.astype(np.int64) - 1, k)


def _expected(prec, s, err="ignore"):
    """Reference module when built (multi-threaded), else the C oracle."""
    dtype = np.float64 if prec == "f64" else np.float32
    mod = oracle.reference_module(prec)
    Gr = s.Gr if s.method != "saft" else np.zeros((0, 3), dtype, order="F")
    if mod is not None:
        return mod.das(s.Y, s.Gt, Gr, s.Ro, dtype(s.dt), s.delay, dtype(s.cp), s.method, err, "cpu", "")
    return oracle.das(s.Y, s.Gt, s.Gr, s.Ro, dtype(s.dt), s.delay, dtype(s.cp), s.method, err, dtype)[0]


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_saft_full_config(prec):
    from dream_b200 import synth
    dtype = np.float64 if prec == "f64" else np.float32
    s = synth.saft_scene(seed=0).astype(dtype)
    assert np.array_equal(_run(prec, s, "stop", "device"), _expected(prec, s, "stop"))


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_tfm_full_config_whole_image(prec):
    """Full TFM configuration (64x64 FMC, K=3000, 512x512): all 262,144 pixels
    of the GPU image equal the reference das / das_f (oracle/_ref, the
    reference's own code; the C oracle when absent) bit for bit."""
    from dream_b200 import synth
    dtype = np.float64 if prec == "f64" else np.float32
    s = synth.tfm_scene(seed=1).astype(dtype)
    Im = _run(prec, s, "stop", "device")
    ref = _expected(prec, s, "stop")
    assert Im.shape == ref.shape == (512 * 512,)
    assert np.array_equal(Im, ref), f"{np.sum(Im != ref)} pixels differ"


@pytest.mark.parametrize("method", ["rca_rowtx", "rca_coltx"])
def test_rca_full_config_z_slabs(method):
    """Full RCA configuration (128x128 row-column array, K=4096, 128x128x256
    grid) in FP32: the whole image on the GPU; three whole 128x128 z-planes
    (49,152 pixels) equal the reference das_f bit for bit."""
    from dream_b200 import synth
    s = synth.rca_scene(seed=2, method=method).astype(np.float32)
    Im = _run("f32", s, "stop", "device")
    sel = rca_slab_points()
    sub = s.astype(np.float32)
    sub.Ro = np.asfortranarray(s.Ro[sel])
    ref = _expected("f32", sub, "stop")
    assert np.array_equal(Im[sel], ref), f"{np.sum(Im[sel] != ref)} pixels differ"


def test_empty_and_degenerate_inputs():
    from dream_b200 import das
    G = np.zeros((2, 3))
    # no observation points
    Im = das.das(np.zeros((10, 4)), G, G, np.zeros((0, 3)), 0.04, 0.0, 1500.0, "tfm", "stop", "cuda")
    assert Im.shape == (0,)
    # zero-length A-scans: every term out of bounds
    Ro = np.array([[0.0, 0.0, 5.0], [1.0, 0.0, 6.0]])
    Im = das.das(np.zeros((0, 4)), G, G, Ro, 0.04, 0.0, 1500.0, "tfm", "ignore", "cuda")
    assert np.array_equal(Im, np.zeros(2))
    with pytest.raises(RuntimeError, match="out-of-bounds"):
        das.das(np.zeros((0, 4)), G, G, Ro, 0.04, 0.0, 1500.0, "tfm", "stop", "cuda")
    # Nr == 0 forces SAFT (extra_src/das.cc:211-213)
    s = build_scene(CASES["saft_f64"])
    a = das.das(s.Y, s.Gt, np.zeros((0, 3)), s.Ro, s.dt, s.delay, s.cp, "tfm", "ignore", "cuda")
    b = das.das(s.Y, s.Gt, None, s.Ro, s.dt, s.delay, s.cp, "saft", "ignore", "cuda")
    assert np.array_equal(a, b)


def test_rca_edge_reads_outside_arrays_rejected():
    from dream_b200 import das
    Gc = np.zeros((20, 3))
    Gr = np.zeros((4, 3))
    with pytest.raises(RuntimeError, match="stripe edges"):
        das.das(np.zeros((10, 80)), Gc, Gr, np.zeros((3, 3)), 0.04, 0.0, 1500.0, "rca", "ignore", "cuda")


def test_cancel_between_launches():
    from dream_b200 import _lib
    L = _lib.load()
    p = _lib.plan_create(_lib.TFM, 100, 10, 2, 2, _lib.PREC_F64, 0)
    p.cancel()
    Y = np.zeros((100, 4), order="F")
    G = np.zeros((2, 3), order="F")
    Ro = np.zeros((10, 3), order="F")
    d = np.zeros(1)
    Im = np.zeros(10)
    ptr = lambda a: a.ctypes.data_as(_lib.ctypes.c_void_p)
    rc = L.dream_das_run(p.handle, ptr(Y), ptr(Ro), ptr(G), ptr(G), 0.04, 0, ptr(d), 1500.0, ptr(Im), 1, None)
    assert rc == _lib.ERR_CANCELLED
    p.set_running()
    rc = L.dream_das_run(p.handle, ptr(Y), ptr(Ro), ptr(G), ptr(G), 0.04, 0, ptr(d), 1500.0, ptr(Im), 1, None)
    assert rc >= 0


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_long_ascans_large_indices(prec):
    """A-scans of 8M samples (dt = 1e-5 us) with indices near 6.7M: the FP32
    kernel truncates through the conversion path for K >= 2^22. Bit-exact
    against the oracle, plain kernels and the FP32-storage kernel."""
    from dream_b200 import synth
    from dream_b200.beamformer import das_mixed
    T = np.float64 if prec == "f64" else np.float32
    rng = np.random.default_rng(12)
    K = 8 << 20
    G = np.asfortranarray(np.array([[-1.0, 0.0, 0.0], [1.5, 0.0, 0.0]]))
    Ro = synth.grid_xz(8, 8, (-3.0, 3.0), (45.0, 55.0))
    Y = np.asfortranarray(rng.normal(size=(K, 4)).astype(T))
    s = synth.Scene(Y, G, G.copy(order="F"), Ro, 1e-5, np.zeros((1, 1)), 1500.0, "tfm", (8, 8)).astype(T)
    ref, st, oob = oracle.das(s.Y, s.Gt, s.Gr, s.Ro, T(s.dt), s.delay, T(s.cp), "tfm", "ignore", T)
    assert oob == 0
    Im = _mod(prec).das(s.Y, s.Gt, s.Gr, s.Ro, T(s.dt), s.delay, T(s.cp), "tfm", "ignore", "cuda")
    assert np.array_equal(Im, ref)
    if prec == "f64":  # FP32 storage with the FP64 indices: the oracle summing the stored samples
        Ys = np.asfortranarray(s.Y.astype(np.float32).astype(np.float64))
        ref32, _, _ = oracle.das(Ys, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", "ignore", np.float64)
        Im32 = das_mixed(s.Y, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", "ignore", "cuda", "f32")
        assert np.abs(Im32 - ref32).max() <= 1e-6 * np.abs(ref32).max()
