"""The allocation-free batch entry point (dream_das_batch_run_noalloc).

It serves callers that cannot call cudaMalloc -- device memory owned by another
framework's pool or a fixed budget, real-time pipelines that forbid allocation
after start-up -- by keeping the batch kernel's scratch (queue counter, frame
table, tile list) in a fixed 4 MiB array inside the library. Through the C ABI
this file checks:

* two calls in a row on uneven TFM and RCA frames (one with a scalar delay, one
  with out-of-bounds terms), with FP32- and BF16-stored A-scans, with a grid hint
  (2-D tiles) and without one (runs of 128 points): every image against the
  oracle summing the same stored samples in FP64 at the reference's FP64 indices
  (1e-6 of max|Im|: a wrong index moves a pixel by O(1)), and against the regular
  batch entry point (dream_das_batch_create + dream_das_batch_run);
* the out-of-bounds count against the oracle's and the batch entry point's;
* rejection of batches beyond the scratch (too many frame descriptors; too many
  tiles);
* refusal of a stream that is being captured into a CUDA graph.

The file name makes pytest collect it last.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _scenes():
    from dream_b200 import synth
    a = synth.tfm_scene(seed=41, n_el=16, K=2000, nx=40, nz=48)
    b = synth.tfm_scene(seed=42, n_el=12, K=900, nx=33, nz=40)  # deep points beyond the A-scans: OOB terms
    b.delay = np.full((1, 1), 0.37, order="F")
    c = synth.rca_scene(seed=43, n_cols=16, n_rows=16, K=4096, nx=8, ny=8, nz=16, method="rca_rowtx")
    d = synth.rca_scene(seed=44, n_cols=12, n_rows=12, K=4096, nx=6, ny=7, nz=10, method="rca_coltx")
    d.delay = np.full((1, 1), 0.11, order="F")
    return [a, b, c, d]


def _stored(Y, storage):
    """The samples the kernel reads, in FP64 (FP32 or BF16 rounding of Y)."""
    t = torch.from_numpy(np.ascontiguousarray(Y, dtype=np.float32))
    if storage == "bf16":
        t = t.to(torch.bfloat16)
    return np.asfortranarray(t.to(torch.float64).numpy())


def _frames(scenes, storage, hinted):
    from dream_b200.batch import make_frame
    from dream_b200.beamformer import grid_hint
    frames = []
    for s in scenes:
        f = make_frame(s.Y, s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, s.method, storage=storage)
        f.n_fast = grid_hint(s.Ro) if hinted else 0
        f.tile = (16, 8) if f.n_fast > 0 else (128, 1)
        f.jc = 16
        frames.append(f)
    return frames


def _structs(frames, outs):
    from dream_b200 import _lib
    from dream_b200.batch import FrameStruct
    from dream_b200.beamformer import parse_method
    arr = (FrameStruct * len(frames))()
    for i, (f, im) in enumerate(zip(frames, outs)):
        arr[i] = FrameStruct(parse_method(f.method), int(f.Y.shape[0]), int(f.Ro.shape[0]), int(f.Gt.shape[0]),
                             int(f.Gr.shape[0]), f.Y.data_ptr(), f.Ro.data_ptr(), f.Gt.data_ptr(), f.Gr.data_ptr(),
                             f.delay.data_ptr(), _lib.DELAY_SINGLE, f.dt, f.cp, im.data_ptr(), int(f.n_fast),
                             int(f.tile[0]), int(f.tile[1]), int(f.jc))
    return arr


def _noalloc(L, arr, n, prec, d_oob, stream):
    return L.dream_das_batch_run_noalloc(ctypes.cast(arr, ctypes.c_void_p), n, prec, torch.cuda.current_device(),
                                         ctypes.c_void_p(d_oob.data_ptr()) if d_oob is not None else None,
                                         ctypes.c_void_p(stream))


@pytest.mark.parametrize("hinted", [True, False], ids=["grid_hint", "no_hint"])
@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_noalloc_matches_oracle_and_batch_entry_point(storage, hinted):
    from dream_b200 import _lib
    from dream_b200.batch import DASBatch
    L = _lib.load()
    scenes = _scenes()
    refs, oob_ref = [], 0
    for s in scenes:
        im, st, oob = oracle.das(_stored(s.Y, storage), s.Gt, s.Gr, s.Ro, s.dt, s.delay, s.cp, s.method, "ignore",
                                 np.float64)
        refs.append(im)
        oob_ref += oob
    assert oob_ref > 0  # the short-A-scan frame has out-of-bounds terms
    frames = _frames(scenes, storage, hinted)
    batch = DASBatch(frames, storage=storage, autotune=False)
    batch.run()
    torch.cuda.synchronize()
    batch_ims = [f.Im.clone() for f in frames]
    assert batch.oob_count() == oob_ref
    prec = _lib.PREC_BF16_STORE if storage == "bf16" else _lib.PREC_F32_STORE
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):  # two calls in a row share (and reuse) the scratch array
        outs = [torch.full_like(f.Im, float("nan")) for f in frames]
        d_oob = torch.zeros(1, dtype=torch.int64, device="cuda")
        rc = _noalloc(L, _structs(frames, outs), len(frames), prec, d_oob, stream)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert int(d_oob.item()) == oob_ref, f"call {call}"
        for i, (o, ref, bim) in enumerate(zip(outs, refs, batch_ims)):
            got = o.cpu().numpy().astype(np.float64)
            scale = np.abs(ref).max()
            assert np.isfinite(got).all(), f"call {call}, frame {i}"
            assert np.abs(got - ref).max() <= 1e-6 * scale, f"call {call}, frame {i}"
            assert float((o - bim).abs().max()) <= 1e-6 * scale, f"call {call}, frame {i}"


def test_noalloc_rejects_too_many_frame_descriptors():
    from dream_b200 import _lib
    from dream_b200.batch import FrameStruct
    L = _lib.load()
    f = _frames(_scenes()[:1], "f32", True)[0]
    im = torch.empty_like(f.Im)
    # 20000 frame descriptors exceed the 4 MiB scratch before any tile is counted
    n = 20000
    arr = (FrameStruct * n)()
    one = _structs([f], [im])[0]
    for i in range(n):
        arr[i] = one
    rc = _noalloc(L, arr, n, _lib.PREC_F32_STORE, None, torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.ERR_ARGUMENT
    assert "4 MiB" in _lib.last_error()


def test_noalloc_rejects_too_many_tiles():
    """One frame of 270,000 tiles of 128 points (more than the tile list fits)
    must be refused. Its buffers are real and sized for the frame, so the
    frame is a valid problem: only the scratch limit refuses it."""
    from dream_b200 import _lib
    from dream_b200.batch import FrameStruct
    L = _lib.load()
    No, K = 128 * 270_000, 16
    Ro = torch.zeros((3, No), dtype=torch.float64, device="cuda").t()
    Y = torch.zeros((1, K), dtype=torch.float32, device="cuda").t()
    G = torch.zeros((3, 1), dtype=torch.float64, device="cuda").t()
    dl = torch.zeros(1, dtype=torch.float64, device="cuda")
    im = torch.empty(No, dtype=torch.float32, device="cuda")
    arr = (FrameStruct * 1)()
    arr[0] = FrameStruct(_lib.TFM, K, No, 1, 1, Y.data_ptr(), Ro.data_ptr(), G.data_ptr(), G.data_ptr(),
                         dl.data_ptr(), _lib.DELAY_SINGLE, 0.04, 1500.0, im.data_ptr(), 0, 128, 1, 16)
    rc = _noalloc(L, arr, 1, _lib.PREC_F32_STORE, None, torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.ERR_ARGUMENT
    msg = _lib.last_error()
    assert "tiles" in msg and "4 MiB" in msg


def test_noalloc_refuses_a_capturing_stream():
    """The frame table is copied from a host array that every call rewrites, so
    a graph captured from a call would beamform whatever the latest call staged:
    the entry point refuses a stream under capture and leaves the capture valid."""
    from dream_b200 import _lib
    L = _lib.load()
    frames = _frames(_scenes()[:1], "f32", True)
    out = torch.empty_like(frames[0].Im)
    arr = _structs(frames, [out])
    d_oob = torch.zeros(1, dtype=torch.int64, device="cuda")
    assert _noalloc(L, arr, 1, _lib.PREC_F32_STORE, d_oob, torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    x = torch.zeros(4, device="cuda")
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            rc = _noalloc(L, arr, 1, _lib.PREC_F32_STORE, d_oob, s.cuda_stream)
            x.add_(1.0)
    torch.cuda.current_stream().wait_stream(s)
    assert rc == _lib.ERR_UNSUPPORTED
    assert "captured" in _lib.last_error()
    g.replay()
    torch.cuda.synchronize()
    assert float(x.sum()) == 4.0  # the capture stayed valid: its one add_ ran on replay
