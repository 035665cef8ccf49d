"""FP32/BF16-storage DAS (precision upgrade) against the FP64 oracle.

Index exactness is checked two ways:
  * index reveal: one element pair and Y[:,0] = k+1 stored exactly in FP32, so
    the image is the selected FP64 index + 1 for every pixel;
  * white-noise A-scans: the oracle sums exactly the same stored (rounded)
    samples in FP64; any wrong index moves a pixel by O(1) while the FP32
    compensated sum stays within 1e-6 of max|Im|.
Image error against the FP64 oracle on the original FP64 A-scans is bounded
by 1e-5 (FP32 storage) and 1e-3 (BF16 storage) relative to max|Im|.
"""
import numpy as np
import pytest

from cases import CASES, _index_reveal, _near_element, build_scene, rca_slab_points
from oracle import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def bf16_round(a):
    t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16).to(torch.float64)
    return np.asfortranarray(t.numpy())


def mixed(s, storage="f32", **kw):
    from dream_b200.beamformer import das_mixed
    Gr = s.Gr if s.method != "saft" else None
    return das_mixed(s.Y, s.Gt, Gr, s.Ro, s.dt, s.delay, s.cp, s.method, kw.pop("err", "ignore"), "cuda",
                     storage, **kw)


def oracle_on_stored(s, storage, err="ignore"):
    Ys = np.asfortranarray(s.Y.astype(np.float32).astype(np.float64)) if storage == "f32" else bf16_round(s.Y)
    return oracle.das(Ys, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, s.method, err, np.float64)


@pytest.mark.parametrize("hint", ["auto", 0])
@pytest.mark.parametrize("grid", [(512, 512, (-20.0, 20.0), (2.0, 50.0)), (96, 96, (-20.0, 20.0), (0.0, 50.0))])
def test_index_reveal_fp64_indices(hint, grid):
    nx, nz, xr, zr = grid
    s = _index_reveal(K=3000, nx=nx, nz=nz, x_rng=xr, z_rng=zr)
    _, _, _, idx = oracle.das(s.Y, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", "ignore", np.float64,
                              return_idx=True)
    Im = mixed(s, hint=hint)
    k = np.where(idx[0] == oracle.OOB_MISS, -1, idx[0])
    assert np.array_equal(Im.astype(np.int64) - 1, k)


@pytest.mark.parametrize("tile", [None, (32, 8), (8, 32)])
@pytest.mark.parametrize("grid", [
    (24, 40, (-20.0, 20.0), (0.0, 50.0), 3000),     # ~43 samples between z neighbours: wide tiles, fast path
    (8, 8, (-20.0, 20.0), (0.0, 400.0), 14000),     # ~1900 samples between neighbours: beyond 4000 per tile
])
def test_index_reveal_coarse_grids(grid, tile):
    """Coarse grids put a leg's samples far apart within one tile (hundreds to
    thousands of samples): the relative fixed point must still select the
    FP64 indices, and tiles spreading beyond its range take the exact path."""
    nx, nz, xr, zr, K = grid
    s = _index_reveal(K=K, nx=nx, nz=nz, x_rng=xr, z_rng=zr)
    _, _, _, idx = oracle.das(s.Y, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", "ignore", np.float64,
                              return_idx=True)
    Im = mixed(s, tile=tile)
    k = np.where(idx[0] == oracle.OOB_MISS, -1, idx[0])
    assert np.array_equal(Im.astype(np.int64) - 1, k)


@pytest.mark.parametrize("delay", [-0.03, -0.045, 0.0])
def test_near_element_truncation(delay):
    s = _near_element(delay)
    ref, st, oob = oracle.das(s.Y, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", "ignore", np.float64)
    Im = mixed(s)
    assert np.array_equal(Im.astype(np.float64), ref)


def test_lattice_exact_integer_times():
    """Distances of 3-4-5 triangles at cp = 1000 m/s and dt = 1 us put many
    products t*Fs on (or within rounding of) integers: the ambiguous-band
    path must reproduce the FP64 truncation."""
    from dream_b200 import synth
    G = np.asfortranarray(np.array([[0.0, 0.0, 0.0], [3.0, 0.0, 0.0], [-4.0, 0.0, 0.0], [6.0, 0.0, 0.0]]))
    xs = np.arange(-12.0, 12.5, 1.0)
    zs = np.arange(0.0, 16.5, 1.0)
    X, Z = np.meshgrid(xs, zs)
    Ro = np.asfortranarray(np.stack([X.flatten("F"), np.zeros(X.size), Z.flatten("F")], 1))
    K = 64
    rng = np.random.default_rng(3)
    Y = np.asfortranarray(rng.normal(size=(K, 16)))
    s = synth.Scene(Y, G, G.copy(order="F"), Ro, 1.0, np.zeros((1, 1)), 1000.0, "tfm", (xs.size, zs.size))
    ref, st, oob = oracle_on_stored(s, "f32")
    Im = mixed(s)
    assert np.abs(Im - ref).max() <= 1e-6 * np.abs(ref).max()
    _, _, oob_g = oracle.das(s.Y, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", "ignore", np.float64)
    assert oob == oob_g


NOISE_CASES = [
    ("tfm", dict(kind="tfm", kw=dict(seed=31, n_el=16, K=3000, nx=40, nz=48))),
    ("tfm_delay", dict(kind="tfm", kw=dict(seed=32, n_el=12, K=3000, nx=33, nz=40), delay=0.41)),
    ("tfm_delayvec", dict(kind="tfm", kw=dict(seed=13, n_el=8, K=3000, nx=16, nz=40), delay_vector_seed=5)),
    ("tfm_oob", dict(kind="tfm", kw=dict(seed=16, n_el=8, K=700, nx=16, nz=16))),
    ("saft", dict(kind="saft", kw=dict(seed=33, n_el=32, K=2048, nx=48, nz=40))),
    ("saft_oob", dict(kind="saft", kw=dict(seed=17, n_el=8, K=400, nx=16, nz=16))),
    ("rca_coltx", dict(kind="rca", kw=dict(seed=34, n_cols=16, n_rows=16, K=4096, nx=8, ny=8, nz=16,
                                           method="rca_coltx"), delay=0.11)),
    ("rca_rowtx", dict(kind="rca", kw=dict(seed=35, n_cols=16, n_rows=16, K=4096, nx=8, ny=8, nz=16,
                                           method="rca_rowtx"), delay=0.11)),
    ("rca_mixed", dict(kind="rca", kw=dict(seed=15, n_cols=8, n_rows=10, K=4096, nx=5, ny=7, nz=6,
                                           method="rca_rowtx"))),
]


@pytest.mark.parametrize("storage", ["f32", "bf16"])
@pytest.mark.parametrize("name,spec", NOISE_CASES, ids=[c[0] for c in NOISE_CASES])
def test_noise_ascans_exact_indices(name, spec, storage):
    s = build_scene(spec)
    rng = np.random.default_rng(99)
    s.Y = np.asfortranarray(rng.normal(size=s.Y.shape))
    ref, st, oob = oracle_on_stored(s, storage)
    Im = mixed(s, storage)
    scale = max(np.abs(ref).max(), 1e-30)
    assert np.abs(Im - ref).max() <= 1e-6 * scale, f"max rel err {np.abs(Im - ref).max() / scale:.3e}"


# FP32 storage: within 1e-5 of max|Im|. BF16 keeps 8 significant bits, so a
# stored sample is off by at most 2^-9 of its magnitude; the per-pixel error is
# bounded by 2^-9 * sum|y| over the selected samples (checked with a factor 2
# for the FP32 sums). Small element counts (the 16-element SAFT, 12x12 RCA
# cases here) keep most of that; the full configurations meet 1e-3 of max|Im|
# (test_tfm_full_config, test_rca_full_config_bf16).
@pytest.mark.parametrize("storage", ["f32", "bf16"])
@pytest.mark.parametrize("name", ["tfm_f64", "saft_f64", "rca_coltx_f64", "rca_rowtx_f64", "tfm_delayvec_f64"])
def test_image_error_vs_fp64_oracle(name, storage):
    s = build_scene(CASES[name])
    ref, _, _ = oracle.das(s.Y, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, s.method, "ignore", np.float64)
    Im = mixed(s, storage)
    if storage == "f32":
        assert np.abs(Im - ref).max() <= 1e-5 * np.abs(ref).max()
    else:
        absum, _, _ = oracle.das(np.abs(s.Y), s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, s.method, "ignore")
        assert np.all(np.abs(Im - ref) <= 2.0 ** -8 * absum + 1e-6 * np.abs(ref).max())


@pytest.mark.parametrize("tile", [(8, 4), (16, 8), (32, 8), (8, 32), (32, 4), (64, 4)])
def test_tile_shapes_same_image(tile):
    s = build_scene(dict(kind="tfm", kw=dict(seed=36, n_el=16, K=3000, nx=40, nz=48)))
    rng = np.random.default_rng(5)
    s.Y = np.asfortranarray(rng.normal(size=s.Y.shape))
    ref, _, _ = oracle_on_stored(s, "f32")
    Im = mixed(s, tile=tile)
    assert np.abs(Im - ref).max() <= 1e-6 * np.abs(ref).max()


def test_unhinted_tiles():
    s = build_scene(dict(kind="tfm", kw=dict(seed=37, n_el=16, K=3000, nx=24, nz=50)))
    rng = np.random.default_rng(6)
    s.Y = np.asfortranarray(rng.normal(size=s.Y.shape))
    ref, _, _ = oracle_on_stored(s, "f32")
    for tile in [None, (64, 1), (32, 1)]:
        Im = mixed(s, hint=0, tile=tile)
        assert np.abs(Im - ref).max() <= 1e-6 * np.abs(ref).max()


def test_oob_levels_and_counts(capsys):
    s = build_scene(dict(kind="tfm", kw=dict(seed=16, n_el=8, K=700, nx=16, nz=16)))
    with pytest.raises(RuntimeError, match="out-of-bounds"):
        mixed(s, err="stop")
    mixed(s, err="warn")
    assert "Warning: DAS out-of-bounds!" in capsys.readouterr().out


def test_weighted_matches_oracle():
    s = build_scene(dict(kind="tfm", kw=dict(seed=38, n_el=8, K=1500, nx=20, nz=30)))
    rng = np.random.default_rng(7)
    s.Y = np.asfortranarray(rng.normal(size=s.Y.shape))
    _, _, _, idx = oracle.das(s.Y, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", "ignore", np.float64,
                              return_idx=True)
    w = rng.uniform(0.2, 1.5, idx.shape[0])
    Ys = s.Y.astype(np.float32).astype(np.float64)
    ref = oracle.weighted(idx, Ys, w.astype(np.float32).astype(np.float64))
    Im = mixed(s, weights=w)
    assert np.abs(Im - ref).max() <= 2e-6 * np.abs(ref).max()


@pytest.fixture(scope="module")
def tfm_full_ref():
    """The TFM configuration and its FP64 image from the reference das
    (oracle/_ref; the C oracle when absent), all 262,144 pixels."""
    from dream_b200 import synth
    s = synth.tfm_scene(seed=1)
    mod = oracle.reference_module("f64")
    if mod is not None:
        ref = mod.das(s.Y, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", "stop", "cpu", "")
    else:
        ref = oracle.das(s.Y, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", "stop")[0]
    return s, ref


@pytest.mark.parametrize("storage,tol", [("f32", 1e-5), ("bf16", 1e-3)])
def test_tfm_full_config(storage, tol, tfm_full_ref):
    """The TFM configuration (64x64 FMC, K=3000, 512x512): the whole image's
    error vs the FP64 reference within tol of max|Im|."""
    s, ref = tfm_full_ref
    Im = mixed(s, storage)
    assert Im.shape == ref.shape
    assert np.abs(Im - ref).max() <= tol * np.abs(ref).max()


@pytest.mark.parametrize("storage,tol", [("f32", 1e-5), ("bf16", 1e-3)])
def test_rca_full_config(storage, tol):
    """RCA configuration (128x128 RCA, K=4096, 128x128x256 grid), FP32 and BF16
    storage: three whole 128x128 z-planes (49,152 pixels) vs the FP64
    reference das within tol of max|Im| (over the planes and the GPU image)."""
    from dream_b200 import synth
    s = synth.rca_scene(seed=2)
    Im = mixed(s, storage)
    sel = rca_slab_points()
    sub = s.astype(np.float64)
    sub.Ro = np.asfortranarray(s.Ro[sel])
    mod = oracle.reference_module("f64")
    if mod is not None:
        ref = mod.das(sub.Y, sub.Gt, sub.Gr, sub.Ro, sub.dt, sub.delay, sub.cp, s.method, "ignore", "cpu", "")
    else:
        ref = oracle.das(sub.Y, sub.Gt, sub.Gr, sub.Ro, sub.dt, sub.delay, sub.cp, s.method, "ignore")[0]
    scale = max(np.abs(Im).max(), np.abs(ref).max())
    assert np.abs(Im[sel] - ref).max() <= tol * scale


@pytest.mark.parametrize("storage", ["f32", "bf16"])
@pytest.mark.parametrize("spec", [
    dict(kind="tfm", kw=dict(seed=71, n_el=40, K=1800, nx=48, nz=40)),
    dict(kind="tfm", kw=dict(seed=74, n_el=41, K=1800, nx=40, nz=36)),
    dict(kind="rca", kw=dict(seed=72, n_cols=32, n_rows=32, K=2600, nx=6, ny=6, nz=10, method="rca_rowtx")),
    dict(kind="rca", kw=dict(seed=73, n_cols=32, n_rows=32, K=2600, nx=6, ny=6, nz=10, method="rca_coltx")),
], ids=["tfm", "tfm_odd", "rca_rowtx", "rca_coltx"])
def test_pipelined_host_upload_matches_device_path(spec, storage):
    """Host arrays (>= 8 MB of A-scans) through the C ABI's host entry
    (dream_das_run), which uploads them in chunks of inner elements (41
    elements: uneven chunk widths) that overlap the beamforming; the image
    equals the device-pointer path's up to the order in which the chunks'
    partial images are added."""
    import ctypes
    from dream_b200 import _lib
    from dream_b200.beamformer import _fast_plan, das_mixed, grid_hint, parse_method
    s = build_scene(spec)
    assert s.Y.nbytes // 2 >= 8 << 20
    Y = np.asfortranarray(s.Y.astype(np.float32))
    f = lambda a: np.asfortranarray(np.asarray(a, dtype=np.float64))
    Gt, Gr, Ro, dl = f(s.Gt), f(s.Gr), f(s.Ro), f(s.delay)
    m = parse_method(s.method)
    prec = _lib.PREC_F32_STORE if storage == "f32" else _lib.PREC_BF16_STORE
    plan = _fast_plan(m, Y.shape[0], Ro.shape[0], Gt.shape[0], Gr.shape[0], prec, 0, grid_hint(Ro))
    host = np.zeros(Ro.shape[0], dtype=np.float32)
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    st = _lib.load().dream_das_run(plan.handle, ptr(Y), ptr(Ro), ptr(Gt), ptr(Gr), s.dt, _lib.DELAY_SINGLE,
                                   ptr(dl), s.cp, ptr(host), _lib.LVL_IGNORE, None)
    assert st >= 0, _lib.last_error()
    t = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64).T)).cuda().t()
    Yd = torch.from_numpy(np.ascontiguousarray(s.Y.astype(np.float32).T)).cuda().t()
    dev = das_mixed(Yd, t(s.Gt), t(s.Gr), t(s.Ro), s.dt, t(s.delay), s.cp, s.method, "ignore", "cuda",
                    storage).cpu().numpy()
    assert np.abs(host - dev).max() <= 2e-6 * np.abs(dev).max()
    ref, _, _ = oracle_on_stored(s, storage)
    assert np.abs(host - ref).max() <= 2e-6 * np.abs(ref).max()


def _run_plan(s, storage, l2_block):
    """FP32/BF16-storage DAS through the C ABI with an explicit L2-blocking
    budget; returns (image, out-of-bounds count, launches)."""
    import ctypes
    from dream_b200 import _lib
    from dream_b200.beamformer import grid_hint, parse_method
    L = _lib.load()
    f = lambda a, dt: torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=dt).T)).cuda().t()
    Y = f(s.Y, np.float32)
    if storage == "bf16":
        Y = Y.t().contiguous().to(torch.bfloat16).t()
    Gt, Gr, Ro, dl = (f(a, np.float64) for a in (s.Gt, s.Gr, s.Ro, s.delay))
    prec = _lib.PREC_F32_STORE if storage == "f32" else _lib.PREC_BF16_STORE
    plan = _lib.plan_create(parse_method(s.method), Y.shape[0], Ro.shape[0], Gt.shape[0], Gr.shape[0], prec, 0)
    _lib.check(L.dream_das_set_grid_hint(plan.handle, grid_hint(s.Ro)))
    _lib.check(L.dream_das_set_l2_block(plan.handle, l2_block))
    Im = torch.empty(Ro.shape[0], dtype=torch.float32, device="cuda")
    oob = torch.zeros(1, dtype=torch.int64, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    _lib.check(L.dream_das_run_device_async(plan.handle, p(Y), p(Ro), p(Gt), p(Gr), s.dt,
                                            _lib.DELAY_MULTIPLE if dl.numel() > 1 else _lib.DELAY_SINGLE, p(dl),
                                            s.cp, p(Im), p(oob), None))
    torch.cuda.synchronize()
    return Im.cpu().numpy(), int(oob.item()), L.dream_das_plan_launch_count(plan.handle)


@pytest.mark.parametrize("storage", ["f32", "bf16"])
@pytest.mark.parametrize("spec", [
    dict(kind="tfm", kw=dict(seed=41, n_el=40, K=2000, nx=24, nz=32)),
    dict(kind="tfm", kw=dict(seed=43, n_el=40, K=700, nx=16, nz=16)),  # out-of-bounds terms
    dict(kind="rca", kw=dict(seed=42, n_cols=40, n_rows=40, K=4096, nx=6, ny=6, nz=12, method="rca_rowtx"),
         delay=0.11),
    dict(kind="rca", kw=dict(seed=44, n_cols=40, n_rows=40, K=4096, nx=6, ny=6, nz=12, method="rca_coltx")),
], ids=["tfm", "tfm_oob", "rca_rowtx", "rca_coltx"])
def test_l2_blocked_passes_match(spec, storage):
    """A-scans beamformed in passes of 16 inner elements (L2 blocking), each
    pass adding into the image: same out-of-bounds count and, up to FP32
    rounding of the pass order, the same image as one pass and as the oracle
    summing the same stored samples."""
    s = build_scene(spec)
    rng = np.random.default_rng(7)
    s.Y = np.asfortranarray(rng.normal(size=s.Y.shape))
    n_out = s.Gt.shape[0] if s.method != "rca_rowtx" else s.Gr.shape[0]
    col_bytes = n_out * s.Y.shape[0] * (4 if storage == "f32" else 2)
    one, oob1, n1 = _run_plan(s, storage, -1)
    blk, oob3, n3 = _run_plan(s, storage, col_bytes * 16)
    assert n3 == 3 * n1  # passes of 16, 16 and 8 inner elements
    assert oob1 == oob3
    ref, _, oob_ref = oracle_on_stored(s, storage)
    scale = max(np.abs(ref).max(), 1e-30)
    assert oob3 == oob_ref
    assert np.abs(blk - ref).max() <= 1e-6 * scale
    assert np.abs(blk - one).max() <= 1e-6 * scale
