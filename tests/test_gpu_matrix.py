"""The beamformer as an explicit sparse matrix (dream_das_indices_device,
dream_b200.matrix): per-term sample indices identical to the oracle's
(the reference's, on every golden case, FP64 and FP32), and row sums in
column order equal to das()/das_f() bit for bit."""
import numpy as np
import pytest

from cases import CASES, build_scene
from oracle import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
scipy_sparse = pytest.importorskip("scipy.sparse")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _scene(name):
    spec = CASES[name]
    T = np.float64 if spec["prec"] == "f64" else np.float32
    return build_scene(spec).astype(T), spec["prec"], T


@pytest.mark.parametrize("name", sorted(CASES))
def test_indices_match_oracle(name):
    from dream_b200.matrix import das_indices
    s, prec, T = _scene(name)
    _, _, oob_ref, idx_ref = oracle.das(s.Y, s.Gt, s.Gr, s.Ro, T(s.dt), s.delay, T(s.cp), s.method, "ignore", T,
                                        return_idx=True)
    Gr = s.Gr if s.method != "saft" else None
    idx, oob = das_indices(s.Gt, Gr, s.Ro, T(s.dt), s.delay, T(s.cp), s.method, s.Y.shape[0], prec)
    ref = np.where(idx_ref == oracle.OOB_MISS, -1, idx_ref)
    assert idx.shape == ref.shape
    assert np.array_equal(idx.cpu().numpy(), ref)
    assert oob == oob_ref


@pytest.mark.parametrize("name", [n for n in sorted(CASES) if "oob_stop" not in n])
def test_row_sums_equal_das(name, golden):
    """CSR rows summed in column order (scipy's sequential product) give the
    reference image bit for bit."""
    from dream_b200.matrix import das_matrix
    g, meta = golden
    s, prec, T = _scene(name)
    Gr = s.Gr if s.method != "saft" else None
    D = das_matrix(s.Gt, Gr, s.Ro, T(s.dt), s.delay, T(s.cp), s.method, s.Y.shape[0], precision=prec,
                   dtype=torch.float64 if prec == "f64" else torch.float32)
    Dh = scipy_sparse.csr_matrix((D.values().cpu().numpy(), D.col_indices().cpu().numpy(),
                                  D.crow_indices().cpu().numpy()), shape=tuple(D.shape))
    C = D.shape[1] // s.Y.shape[0]
    Im = Dh @ np.asarray(s.Y[:, :C], dtype=T).reshape(-1, order="F")
    ref = g[name + "__Im"]
    assert Im.dtype == ref.dtype
    assert np.array_equal(Im, ref)


def test_weighted_matrix_and_device_product():
    """Per-column weights, the product on the device (cuSPARSE), and the
    adjoint D^T x against the oracle's index-table operators."""
    from dream_b200.matrix import das_indices, das_matrix
    s, _, _ = _scene("tfm_f64")
    rng = np.random.default_rng(4)
    C = s.Gt.shape[0] * s.Gr.shape[0]
    w = rng.uniform(0.5, 1.5, C)
    D = das_matrix(s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", s.Y.shape[0], weights=w)
    idx, _ = das_indices(s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, "tfm", s.Y.shape[0])
    idx = idx.cpu().numpy()
    y = torch.from_numpy(s.Y.reshape(-1, order="F")).cuda()
    Im = torch.mv(D, y).cpu().numpy()
    ref = oracle.weighted(idx, s.Y, w)
    assert np.abs(Im - ref).max() <= 1e-12 * np.abs(ref).max()
    x = rng.normal(size=s.Ro.shape[0])
    Ya = torch.mv(D.to_sparse_coo().t().to_sparse_csr(), torch.from_numpy(x).cuda()).cpu().numpy()
    Ya_ref = oracle.adjoint(idx, x, w, s.Y.shape[0]).reshape(-1, order="F")
    assert np.abs(Ya - Ya_ref).max() <= 1e-12 * np.abs(Ya_ref).max()
