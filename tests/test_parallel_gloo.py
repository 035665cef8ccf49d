"""Multi-rank DAS logic on CPU ranks (torch.distributed gloo, world size 2):
transmit, inner-element and image-point shards of the forward, inner-element
shards of the adjoint.

The per-rank compute is the oracle here (the sharding and collectives are what
is tested); on GPUs the same functions run with dream_b200.parallel.cuda_compute
over NCCL. Includes a failure case: a rank that dies before the collective makes
the survivor's all-reduce fail within the process-group timeout.
"""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _oracle_compute(Y, Gt, Gr, Ro, dt, delay, cp, method):
    sys.path.insert(0, ROOT)
    from oracle import oracle
    Im, _, _ = oracle.das(np.asarray(Y), np.asarray(Gt), np.asarray(Gr), np.asarray(Ro), dt, delay, cp, method,
                          "ignore", np.float64)
    return torch.from_numpy(Im)


def _oracle_inner_compute(Y_local, Gt, Gr, Ro, dt, delay, cp, method, inner):
    """Partial image over inner elements [lo, hi) from a shard's A-scans, at the
    oracle's indices (every term of those columns)."""
    sys.path.insert(0, ROOT)
    from dream_b200.parallel import element_counts
    from oracle import oracle
    Gt, Gr, Ro = np.asarray(Gt), np.asarray(Gr), np.asarray(Ro)
    n_out, n_in = element_counts(method, Gt.shape[0], Gr.shape[0])
    K = np.asarray(Y_local).shape[0]
    _, _, _, idx = oracle.das(np.zeros((K, n_out * n_in)), Gt, Gr, Ro, dt, delay, cp, method, "ignore",
                              np.float64, return_idx=True)
    lo, hi = inner
    Yl = np.asarray(Y_local)
    Im = np.zeros(Ro.shape[0])
    for o in range(n_out):
        for i in range(lo, hi):
            k = idx[o * n_in + i]
            ok = k != oracle.OOB_MISS
            Im[ok] += Yl[k[ok], o * (hi - lo) + i - lo]
    return torch.from_numpy(Im)


def _oracle_adjoint_compute(x, Gt, Gr, Ro, dt, delay, cp, method, K, inner):
    """The shard's A-scan columns of DAS^T x at the oracle's indices."""
    sys.path.insert(0, ROOT)
    from dream_b200.parallel import inner_columns
    from oracle import oracle
    Gt, Gr, Ro = np.asarray(Gt), np.asarray(Gr), np.asarray(Ro)
    cols = inner_columns(method, Gt.shape[0], Gr.shape[0], *inner)
    n = Gt.shape[0] * Gr.shape[0]
    _, _, _, idx = oracle.das(np.zeros((K, n)), Gt, Gr, Ro, dt, delay, cp, method, "ignore", np.float64,
                              return_idx=True)
    return torch.from_numpy(oracle.adjoint(idx[cols], x.numpy().astype(np.float64), np.ones(cols.size), K))


def _worker(rank, world, port, mode, spec, out_dir):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    from cases import build_scene
    from dream_b200 import parallel
    s = build_scene(spec)
    try:
        if mode == "tx":
            lo, hi = parallel.block_range(s.Gt.shape[0], world, rank)
            c0, c1 = parallel.tx_columns(s.method, s.Gt.shape[0], s.Gr.shape[0], lo, hi)
            Im = parallel.das_shard_tx(_oracle_compute, s.Y[:, c0:c1], s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp,
                                       s.method)
        elif mode == "inner":
            n_out, n_in = parallel.element_counts(s.method, s.Gt.shape[0], s.Gr.shape[0])
            lo, hi = parallel.block_range(n_in, world, rank)
            cols = parallel.inner_columns(s.method, s.Gt.shape[0], s.Gr.shape[0], lo, hi)
            Im = parallel.das_shard_inner(_oracle_inner_compute, np.asfortranarray(s.Y[:, cols]), s.Gt, s.Gr, s.Ro,
                                          s.dt, s.delay, s.cp, s.method)
        elif mode == "adjoint":
            x = torch.from_numpy(np.random.default_rng(9).normal(size=s.Ro.shape[0])) if rank == 0 \
                else torch.zeros(s.Ro.shape[0], dtype=torch.float64)
            Ya = parallel.das_adjoint_shard_inner(_oracle_adjoint_compute, x, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp,
                                                  s.method, s.Y.shape[0])
            np.save(os.path.join(out_dir, f"r{rank}.npy"), Ya.numpy())
            return
        elif mode == "pixels":
            Im = parallel.das_shard_pixels(_oracle_compute, s.Y, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, s.method)
        elif mode == "rank_dies":
            if rank == 1:
                os._exit(3)  # leaves between steps, before the collective
            t = torch.ones(4)
            try:
                dist.all_reduce(t)
                np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array([0.0]))
            except Exception:
                np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array([1.0]))  # failure detected
            return
        np.save(os.path.join(out_dir, f"r{rank}.npy"), Im.numpy())
    finally:
        if mode != "rank_dies":
            dist.destroy_process_group()


def _run(mode, spec, tmp_path, world=2):
    port = _port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, port, mode, spec, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    return [np.load(tmp_path / f"r{r}.npy") if (tmp_path / f"r{r}.npy").exists() else None for r in range(world)]


def _full(spec):
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from cases import build_scene
    from oracle import oracle
    s = build_scene(spec)
    return oracle.das(s.Y, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, s.method, "ignore", np.float64)[0]


TFM = dict(kind="tfm", kw=dict(seed=51, n_el=7, K=1500, nx=9, nz=13))


def test_tx_sharded_tfm_equals_full_image(tmp_path):
    out = _run("tx", TFM, tmp_path)
    ref = _full(TFM)
    for Im in out:
        # partial images add in a different order than the reference's single sum
        assert np.abs(Im - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.array_equal(out[0], out[1])


INNER_SPECS = [
    TFM,
    dict(kind="rca", kw=dict(seed=54, n_cols=7, n_rows=7, K=2500, nx=3, ny=4, nz=5, method="rca_rowtx")),
    dict(kind="rca", kw=dict(seed=55, n_cols=6, n_rows=6, K=2500, nx=4, ny=3, nz=5, method="rca_coltx")),
]


@pytest.mark.parametrize("spec", INNER_SPECS, ids=["tfm", "rca_rowtx", "rca_coltx"])
def test_inner_sharded_equals_full_image(spec, tmp_path):
    """Each rank holds the A-scans of its block of inner elements (RCA: the
    stripes of one direction) and the full element arrays; one all-reduce of
    the partial images gives the unsharded image within 1e-12 relative."""
    out = _run("inner", spec, tmp_path)
    ref = _full(spec)
    for Im in out:
        assert np.abs(Im - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("spec", INNER_SPECS, ids=["tfm", "rca_rowtx", "rca_coltx"])
def test_adjoint_inner_shards_assemble_the_full_adjoint(spec, tmp_path):
    """x broadcast from rank 0, every rank writes the columns of its inner
    block: put together, the columns are the unsharded adjoint's."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from cases import build_scene
    from dream_b200 import parallel
    from oracle import oracle
    out = _run("adjoint", spec, tmp_path)
    s = build_scene(spec)
    x = np.random.default_rng(9).normal(size=s.Ro.shape[0])
    n = s.Gt.shape[0] * s.Gr.shape[0]
    K = s.Y.shape[0]
    _, _, _, idx = oracle.das(np.zeros((K, n)), s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, s.method, "ignore",
                              np.float64, return_idx=True)
    full = oracle.adjoint(idx, x, np.ones(n), K)
    n_out, n_in = parallel.element_counts(s.method, s.Gt.shape[0], s.Gr.shape[0])
    for r, Ya in enumerate(out):
        lo, hi = parallel.block_range(n_in, 2, r)
        cols = parallel.inner_columns(s.method, s.Gt.shape[0], s.Gr.shape[0], lo, hi)
        assert np.array_equal(Ya, full[:, cols])


def test_inner_columns_partition_every_column():
    from dream_b200.parallel import block_range, inner_columns
    for method, Nt, Nr in (("tfm", 5, 7), ("rca_rowtx", 6, 4), ("rca_coltx", 3, 8)):
        for world in (1, 2, 3):
            n_in = Nt if method == "rca_rowtx" else Nr
            cols = np.concatenate([inner_columns(method, Nt, Nr, *block_range(n_in, world, r)) for r in range(world)])
            assert np.array_equal(np.sort(cols), np.arange(Nt * Nr))


@pytest.mark.parametrize("spec", [
    TFM,
    dict(kind="rca", kw=dict(seed=52, n_cols=6, n_rows=6, K=2500, nx=3, ny=4, nz=5, method="rca_rowtx")),
    dict(kind="saft", kw=dict(seed=53, n_el=9, K=2048, nx=7, nz=11)),
])
def test_pixel_sharded_equals_full_image_exactly(spec, tmp_path):
    out = _run("pixels", spec, tmp_path)
    ref = _full(spec)
    for Im in out:
        assert np.array_equal(Im, ref)


def test_block_ranges_cover_uneven_counts():
    from dream_b200.parallel import block_range
    for n in (0, 1, 7, 64, 101):
        for w in (1, 2, 3, 8):
            rs = [block_range(n, w, r) for r in range(w)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            assert max(h - l for l, h in rs) - min(h - l for l, h in rs) <= 1


def test_rank_failure_is_detected_by_the_survivor(tmp_path):
    out = _run("rank_dies", TFM, tmp_path)
    assert out[1] is None
    assert out[0] is not None and out[0][0] == 1.0
