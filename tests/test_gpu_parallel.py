"""The sharded paths with the CUDA compute on one GPU (NCCL, world size 1):
the same code the multi-GPU run executes, checked against the one-call image."""
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
