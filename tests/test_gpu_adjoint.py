"""Differentiable DAS: the CUDA gather/scatter/weight-gradient operators
against the FP64 oracle on explicit index tables, the dot-product test,
finite differences and a CPU reference gradient, and the CG reconstruction."""
import numpy as np
import pytest

from cases import build_scene
from oracle import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def das_scatter(x, w, op):
    from dream_b200.autograd import das_scatter as f
    return f(x, w, op)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _setup(method="tfm", seed=41, **kw):
    if method == "tfm":
        s = build_scene(dict(kind="tfm", kw=dict(seed=seed, n_el=8, K=900, nx=20, nz=24, **kw)))
    else:
        s = build_scene(dict(kind="rca", kw=dict(seed=seed, n_cols=8, n_rows=8, K=2500, nx=5, ny=6, nz=8,
                                                 method=method)))
    from dream_b200.autograd import DASOperator
    op = DASOperator(s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, s.method, s.Y.shape[0])
    _, _, _, idx = oracle.das(s.Y, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, s.method, "ignore", np.float64,
                              return_idx=True)
    return s, op, idx


def f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


@pytest.mark.parametrize("method", ["tfm", "rca_coltx", "rca_rowtx"])
def test_operators_match_oracle(method):
    s, op, idx = _setup(method)
    rng = np.random.default_rng(1)
    C, No = idx.shape
    K = s.Y.shape[0]
    Y = f32(rng.normal(size=(K, C)))
    w = f32(rng.uniform(0.3, 1.2, C))
    x = f32(rng.normal(size=No))
    Yt = torch.from_numpy(np.ascontiguousarray(Y.T)).float().cuda().t()
    wt = torch.from_numpy(w).float().cuda()
    xt = torch.from_numpy(x).float().cuda()
    Im = op.forward(Yt, wt).cpu().double().numpy()
    ref = oracle.weighted(idx, Y, w)
    assert np.abs(Im - ref).max() <= 2e-6 * np.abs(ref).max()
    Ya = op.adjoint(xt, wt).cpu().double().numpy()
    refa = oracle.adjoint(idx, x, w, K)
    assert np.abs(Ya - refa).max() <= 1e-5 * np.abs(refa).max()
    dw = op.wgrad(xt, Yt).cpu().double().numpy()
    refw = oracle.wgrad(idx, x, Y)
    assert np.abs(dw - refw).max() <= 1e-5 * np.abs(refw).max()
    Yg, dw2 = op.backward(xt, Yt, wt)
    assert torch.allclose(Yg, op.adjoint(xt, wt), rtol=1e-5, atol=1e-5 * float(np.abs(refa).max()))
    assert torch.allclose(dw2, op.wgrad(xt, Yt), rtol=1e-5, atol=1e-5 * float(np.abs(refw).max()))


def test_adjoint_lattice_exact_integer_times():
    """A lattice of 3-4-5 triangles (cp = 1000 m/s, dt = 1 us) puts many
    terms' sample positions on, or within rounding of, integers. In the
    adjoint those terms take the ambiguous-band path: the window additions of
    their (outer element, chunk) batch are taken back out and the exact FP64
    indices used instead, so every term must still land where the oracle's
    index puts it (adjoint and weight gradient)."""
    from dream_b200.autograd import DASOperator
    G = np.asfortranarray(np.array([[0.0, 0.0, 0.0], [3.0, 0.0, 0.0], [-4.0, 0.0, 0.0], [6.0, 0.0, 0.0]]))
    xs = np.arange(-12.0, 12.5, 1.0)
    zs = np.arange(0.0, 16.5, 1.0)
    X, Z = np.meshgrid(xs, zs)
    Ro = np.asfortranarray(np.stack([X.flatten("F"), np.zeros(X.size), Z.flatten("F")], 1))
    K, dl = 64, np.zeros((1, 1))
    rng = np.random.default_rng(7)
    Y = f32(rng.normal(size=(K, 16)))
    _, _, _, idx = oracle.das(np.asfortranarray(Y), G, G, Ro, 1.0, dl, 1000.0, "tfm", "ignore", np.float64,
                              return_idx=True)
    op = DASOperator(G, G.copy(order="F"), Ro, 1.0, dl, 1000.0, "tfm", K)
    C, No = idx.shape
    w = f32(rng.uniform(0.3, 1.2, C))
    x = f32(rng.normal(size=No))
    Yt = torch.from_numpy(np.ascontiguousarray(Y.T)).float().cuda().t()
    wt = torch.from_numpy(w).float().cuda()
    xt = torch.from_numpy(x).float().cuda()
    Ya = op.adjoint(xt, wt).cpu().double().numpy()
    refa = oracle.adjoint(idx, x, w, K)
    assert np.abs(Ya - refa).max() <= 1e-5 * np.abs(refa).max()
    dw = op.wgrad(xt, Yt).cpu().double().numpy()
    refw = oracle.wgrad(idx, x, Y)
    assert np.abs(dw - refw).max() <= 1e-5 * np.abs(refw).max()


def test_dot_product_full_cg_config():
    """<DAS_w Y, x> = <Y, DAS_w^T x> on the 32x32, K=2048, 256x256 configuration."""
    from dream_b200 import synth
    from dream_b200.autograd import DASOperator
    s = synth.cg_scene(seed=4)
    op = DASOperator(s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", 2048)
    g = torch.Generator(device="cuda").manual_seed(0)
    Y = torch.randn(op.ncol, op.K, device="cuda", generator=g).t()
    x = torch.randn(op.No, device="cuda", generator=g)
    w = torch.rand(op.ncol, device="cuda", generator=g) + 0.5
    lhs = torch.dot(op.forward(Y, w).double(), x.double())
    rhs = torch.sum(Y.double() * op.adjoint(x, w).double())
    assert abs(float(lhs - rhs)) <= 1e-5 * abs(float(lhs))


def _loss(op, x, w, Y, lam):
    R = das_scatter(x, w, op)
    return ((R.double() - Y.double()) ** 2).sum() + lam * (x.double() ** 2).sum()


GRAD_CONFIGS = {
    # a reduced problem: 8 x 8 elements, 32 x 32 image
    "reduced_8x8_32x32": dict(seed=6, n_el=8, K=1024, nx=32, nz=32, density=0.05, x_rng=(-4.0, 4.0),
                              z_rng=(5.0, 15.0)),
    # the model-based reconstruction configuration: 32 x 32 elements, K = 2048, 256 x 256 image
    "cg_32x32_K2048_256x256": dict(seed=4),
}


@pytest.mark.parametrize("cfg", sorted(GRAD_CONFIGS))
def test_gradients_fd_and_cpu_reference(cfg):
    """Gradients of ||DAS_w^T x - Y||^2 + lam||x||^2 w.r.t. x and w: autograd vs
    central finite differences (h = 1e-3) on 6 weights and 6 image points, and
    vs the FP64 CPU reference on the oracle's index table."""
    from dream_b200 import synth
    from dream_b200.autograd import DASOperator
    s = synth.cg_scene(**GRAD_CONFIGS[cfg])
    K = s.Y.shape[0]
    op = DASOperator(s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", K)
    _, _, _, idx = oracle.das(np.zeros((K, op.ncol)), s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", "ignore",
                              np.float64, return_idx=True)
    lam = 1e-3
    rng = np.random.default_rng(2)
    x0 = f32(s.extra["reflectivity"] + 0.1 * rng.normal(size=op.No))
    w0 = f32(rng.uniform(0.5, 1.5, op.ncol))
    Ytrue = oracle.adjoint(idx, s.extra["reflectivity"], np.ones(op.ncol), K)
    Ynp = f32(Ytrue + 0.01 * rng.normal(size=Ytrue.shape))
    Y = torch.from_numpy(np.ascontiguousarray(Ynp.T)).float().cuda().t()
    x = torch.from_numpy(x0).float().cuda().requires_grad_(True)
    w = torch.from_numpy(w0).float().cuda().requires_grad_(True)
    L = _loss(op, x, w, Y, lam)
    gx, gw = torch.autograd.grad(L, (x, w))
    gx, gw = gx.double().cpu().numpy(), gw.double().cpu().numpy()
    # CPU reference (FP64 on the oracle index table)
    R = oracle.adjoint(idx, x0, w0, K) - Ynp
    ref_gx = 2.0 * oracle.weighted(idx, R, w0) + 2.0 * lam * x0
    ref_gw = 2.0 * oracle.wgrad(idx, x0, R)
    assert np.abs(gx - ref_gx).max() <= 1e-4 * np.abs(ref_gx).max()
    assert np.abs(gw - ref_gw).max() <= 1e-4 * np.abs(ref_gw).max()
    # Central finite differences, h = 1e-3. Perturbing w[c] changes only column c
    # of DAS_w^T x, and x[n] only the samples k(n, c'); every other term of the
    # loss is equal in exact arithmetic at w +- e and x +- e, so each difference
    # is summed over the touched entries (plus the regulariser): the same
    # derivative, without the FP32 rounding of the untouched entries, which
    # depends on the order of the scatter's additions and would swamp the
    # 2*h*grad difference on the full configuration.
    h = 1e-3
    Yd = Y.double()
    with torch.no_grad():
        for c in rng.choice(op.ncol, 6, replace=False):
            e = torch.zeros_like(w)
            e[c] = h
            Lc = lambda ww: float(((das_scatter(x, ww, op)[:, c].double() - Yd[:, c]) ** 2).sum())
            fd = (Lc(w + e) - Lc(w - e)) / (2 * h)
            assert abs(fd - gw[c]) <= 2e-3 * max(abs(gw[c]), 1e-3 * np.abs(gw).max())
        for n in rng.choice(op.No, 6, replace=False):
            e = torch.zeros_like(x)
            e[n] = h
            cols = np.nonzero(idx[:, n] != oracle.OOB_MISS)[0]
            ks = torch.from_numpy(idx[cols, n]).cuda()
            cs = torch.from_numpy(cols).cuda()

            def Ln(xx):
                R = das_scatter(xx, w, op)[ks, cs].double() - Yd[ks, cs]
                return float((R ** 2).sum()) + lam * float((xx.double()[n]) ** 2)
            fd = (Ln(x + e) - Ln(x - e)) / (2 * h)
            assert abs(fd - gx[n]) <= 2e-3 * max(abs(gx[n]), 1e-3 * np.abs(gx).max())


def test_gather_autograd_matches_adjoint():
    s, op, idx = _setup("tfm", seed=43)
    from dream_b200.autograd import das_gather
    rng = np.random.default_rng(3)
    Y = torch.randn(op.ncol, op.K, device="cuda").t().requires_grad_(True)
    w = torch.rand(op.ncol, device="cuda").requires_grad_(True)
    g = torch.randn(op.No, device="cuda")
    Im = das_gather(Y, w, op)
    gY, gw = torch.autograd.grad(Im, (Y, w), grad_outputs=g)
    assert torch.allclose(gY, op.adjoint(g, w.detach()), atol=1e-5)
    assert torch.allclose(gw, op.wgrad(g, Y.detach()), rtol=1e-5, atol=1e-4)


def test_cg_reconstruction_converges():
    """30 CG iterations on the 32x32 / K=2048 / 256x256 configuration."""
    from dream_b200 import synth
    from dream_b200.autograd import DASOperator, cg_reconstruct
    s = synth.cg_scene(seed=4)
    op = DASOperator(s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", 2048)
    xt = torch.from_numpy(s.extra["reflectivity"]).float().cuda()
    w = torch.ones(op.ncol, device="cuda")
    Y = op.adjoint(xt, w)
    x, res = cg_reconstruct(op, Y, w, lam=1e-3, iters=30)
    # the normal equations are ill-conditioned (lam is small against the
    # operator norm): require a 10x residual reduction and a reconstruction
    # that matches the true reflectivity
    assert float(res[-1]) < 0.1 * float(res[0])
    corr = float(torch.dot(x, xt) / (x.norm() * xt.norm()))
    assert corr > 0.5, corr


def test_cg_graph_replay_matches_eager():
    """The CG solve captured in a CUDA graph gives the eager result, and a
    replay after writing new A-scans into the static buffer re-solves."""
    from dream_b200 import synth
    from dream_b200.autograd import CGGraph, DASOperator, cg_reconstruct
    s = synth.cg_scene(seed=8, n_el=16, K=1024, nx=64, nz=64, x_rng=(-4.0, 4.0), z_rng=(5.0, 20.0))
    op = DASOperator(s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", 1024)
    xt = torch.from_numpy(s.extra["reflectivity"]).float().cuda()
    w = torch.ones(op.ncol, device="cuda")
    Y = op.adjoint(xt, w)
    x_e, r_e = cg_reconstruct(op, Y, w, 1e-3, 10)
    g = CGGraph(op, Y, w, 1e-3, 10)
    x_g, r_g = g.replay()
    torch.cuda.synchronize()
    assert torch.allclose(x_g, x_e, rtol=1e-4, atol=1e-5 * float(x_e.abs().max()))
    g.Y.copy_(2.0 * Y)
    x_2, _ = g.replay()
    torch.cuda.synchronize()
    assert torch.allclose(x_2, 2.0 * x_e, rtol=1e-3, atol=1e-4 * float(x_e.abs().max()))
