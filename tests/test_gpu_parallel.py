"""The sharded paths with the CUDA compute on one GPU (NCCL, world size 1):
the same code the multi-GPU run executes, checked against the one-call image;
inner-element shards of the forward and the adjoint on the device."""
import datetime
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_cuda_compute_sharded_world1():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import torch.distributed as dist
    from cases import build_scene
    from dream_b200 import parallel
    from dream_b200.beamformer import das_mixed
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sc = build_scene(dict(kind="tfm", kw=dict(seed=61, n_el=8, K=1500, nx=24, nz=32)))
        comp = parallel.cuda_compute("f32")
        ref = das_mixed(sc.Y, sc.Gt, sc.Gr, sc.Ro, sc.dt, sc.delay, sc.cp, "tfm", "ignore", "cuda", "f32")
        a = parallel.das_shard_tx(comp, sc.Y, sc.Gt, sc.Gr, sc.Ro, sc.dt, sc.delay, sc.cp, "tfm").cpu().numpy()
        b = parallel.das_shard_pixels(comp, sc.Y, sc.Gt, sc.Gr, sc.Ro, sc.dt, sc.delay, sc.cp, "tfm").cpu().numpy()
        assert np.array_equal(a, ref) and np.array_equal(b, ref)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("method", ["tfm", "rca_rowtx", "rca_coltx"])
def test_inner_shards_add_up_to_the_frame(method):
    """The partial images of two inner-element shards (A-scans holding only
    the shard's columns, full element arrays) add up to the unsharded image,
    and each shard's adjoint columns equal the unsharded adjoint's."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cases import build_scene
    from dream_b200 import parallel
    from dream_b200.autograd import DASOperator
    from dream_b200.beamformer import das_mixed
    if method == "tfm":
        sc = build_scene(dict(kind="tfm", kw=dict(seed=62, n_el=9, K=1500, nx=24, nz=32)))
    else:
        sc = build_scene(dict(kind="rca", kw=dict(seed=63, n_cols=10, n_rows=10, K=2600, nx=6, ny=5, nz=8,
                                                  method=method)))
    Nt, Nr = sc.Gt.shape[0], sc.Gr.shape[0]
    n_out, n_in = parallel.element_counts(method, Nt, Nr)
    full = das_mixed(sc.Y, sc.Gt, sc.Gr, sc.Ro, sc.dt, sc.delay, sc.cp, method, "ignore", "cuda", "f32")
    parts = []
    for r in range(2):
        lo, hi = parallel.block_range(n_in, 2, r)
        cols = parallel.inner_columns(method, Nt, Nr, lo, hi)
        Yl = torch.from_numpy(np.ascontiguousarray(sc.Y[:, cols].T, dtype=np.float32)).cuda().t()
        parts.append(das_mixed(Yl, sc.Gt, sc.Gr, sc.Ro, sc.dt, sc.delay, sc.cp, method, "ignore", "cuda", "f32",
                               inner=(lo, hi)).cpu().numpy())
    scale = np.abs(full).max()
    assert np.abs(parts[0] + parts[1] - full).max() <= 1e-6 * scale
    # adjoint: each shard's columns
    x = torch.from_numpy(np.random.default_rng(4).normal(size=sc.Ro.shape[0])).float().cuda()
    op = DASOperator(sc.Gt, sc.Gr, sc.Ro, sc.dt, sc.delay, sc.cp, method, sc.Y.shape[0])
    Ya = op.adjoint(x).cpu().numpy()
    for r in range(2):
        lo, hi = parallel.block_range(n_in, 2, r)
        cols = parallel.inner_columns(method, Nt, Nr, lo, hi)
        ops = DASOperator(sc.Gt, sc.Gr, sc.Ro, sc.dt, sc.delay, sc.cp, method, sc.Y.shape[0], inner=(lo, hi))
        Ys = ops.adjoint(x).cpu().numpy()
        assert Ys.shape == (sc.Y.shape[0], cols.size)
        assert np.abs(Ys - Ya[:, cols]).max() <= 1e-5 * np.abs(Ya).max()
