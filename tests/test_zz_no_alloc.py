"""The allocation-free batch entry point (dream_das_batch_run_noalloc).

It serves callers that cannot call cudaMalloc -- device memory owned by another
framework's pool or a fixed budget, real-time pipelines that forbid allocation
after start-up -- by keeping the batch kernel's scratch (queue counter, frame
table, tile list) in a fixed 4 MiB array inside the library. This test calls it
through the C ABI twice in a row and checks both outputs against the regular
batch entry point (dream_das_batch_create + dream_das_batch_run) on the same
frames, with the same tiles, within 1e-6 of max|Im|. The file name makes
pytest collect it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _frames():
    from dream_b200 import synth
    from dream_b200.batch import make_frame
    frames = []
    for sp in synth.batch_specs(21, 4):
        sp = dict(sp, side=min(sp["side"], 96), n_el=min(sp["n_el"], 32))
        Y, G, Ro, dt, cp = synth.tfm_frame_torch(sp)
        f = make_frame(Y, G, G, Ro, dt, np.zeros((1, 1)), cp, "tfm")
        f.tile, f.jc = (16, 8), 16
        frames.append(f)
    return frames


def _structs(frames, outs):
    from dream_b200 import _lib
    from dream_b200.batch import FrameStruct
    from dream_b200.beamformer import grid_hint
    arr = (FrameStruct * len(frames))()
    for i, (f, im) in enumerate(zip(frames, outs)):
        arr[i] = FrameStruct(_lib.TFM, int(f.Y.shape[0]), int(f.Ro.shape[0]), int(f.Gt.shape[0]), int(f.Gr.shape[0]),
                             f.Y.data_ptr(), f.Ro.data_ptr(), f.Gt.data_ptr(), f.Gr.data_ptr(), f.delay.data_ptr(),
                             _lib.DELAY_SINGLE, f.dt, f.cp, im.data_ptr(), grid_hint(f.Ro), 16, 8, 16)
    return arr


def test_noalloc_batch_matches_batch_entry_point():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dream_b200 import _lib
    from dream_b200.batch import DASBatch
    L = _lib.load()
    frames = _frames()
    ref_batch = DASBatch(frames, autotune=False)
    ref_batch.run()
    torch.cuda.synchronize()
    refs = [f.Im.clone() for f in frames]
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    d_oob = torch.zeros(1, dtype=torch.int64, device="cuda")
    for call in range(2):  # two calls in a row share (and reuse) the scratch array
        outs = [torch.full_like(r, float("nan")) for r in refs]
        arr = _structs(frames, outs)
        rc = L.dream_das_batch_run_noalloc(ctypes.cast(arr, ctypes.c_void_p), len(frames), _lib.PREC_F32_STORE,
                                           torch.cuda.current_device(), ctypes.c_void_p(d_oob.data_ptr()), stream)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        for r, o in zip(refs, outs):
            scale = float(r.abs().max())
            assert bool(torch.isfinite(o).all())
            assert float((o - r).abs().max()) <= 1e-6 * scale, f"call {call}"


def test_noalloc_rejects_batches_beyond_its_scratch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dream_b200 import _lib
    from dream_b200.batch import FrameStruct
    L = _lib.load()
    f = _frames()[0]
    im = torch.empty_like(f.Im)
    # 20000 frames of descriptors exceed the 4 MiB scratch before any tile is counted
    n = 20000
    arr = (FrameStruct * n)()
    one = _structs([f], [im])[0]
    for i in range(n):
        arr[i] = one
    rc = L.dream_das_batch_run_noalloc(ctypes.cast(arr, ctypes.c_void_p), n, _lib.PREC_F32_STORE,
                                       torch.cuda.current_device(), None,
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.ERR_ARGUMENT
    assert "4 MiB" in _lib.last_error()
