"""Batched DAS: one persistent launch over uneven frames (and its CUDA graph)
against the reference's FP64 image of the same stored samples, and the
per-frame FP32-storage kernel; the autotuner's choices are valid."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda(tmp_path_factory):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import os
    os.environ["DREAM_AUTOTUNE_CACHE"] = str(tmp_path_factory.mktemp("tune") / "autotune.json")


def _frames(n=6, seed=11, max_side=160, storage="f32"):
    from dream_b200 import synth
    from dream_b200.batch import make_frame
    specs = synth.batch_specs(seed, n)
    frames = []
    for sp in specs:
        sp = dict(sp, side=min(sp["side"], max_side))
        Y, G, Ro, dt, cp = synth.tfm_frame_torch(sp)
        frames.append(make_frame(Y, G, G, Ro, dt, np.zeros((1, 1)), cp, "tfm", storage=storage))
    return frames


def _expected(f, storage):
    """The frame's image from the reference das (oracle/_ref; the C oracle when
    absent) on exactly the stored samples (FP32 or BF16 values in FP64), so
    every sum is exact and every index is the reference's FP64 index."""
    from oracle import oracle
    Ys = np.asfortranarray(f.Y.float().t().contiguous().t().cpu().numpy().astype(np.float64))
    args = [np.asfortranarray(a.cpu().numpy()) for a in (f.Gt, f.Gr, f.Ro, f.delay)]
    mod = oracle.reference_module("f64")
    if mod is not None:
        return mod.das(Ys, args[0], args[1], args[2], f.dt, args[3], f.cp, f.method, "ignore", "cpu", "")
    return oracle.das(Ys, args[0], args[1], args[2], f.dt, args[3], f.cp, f.method, "ignore", np.float64)[0]


def _single(f, storage):
    """The one-frame kernel on the same stored samples."""
    from dream_b200.beamformer import das_mixed
    Y = f.Y.float() if storage == "bf16" else f.Y
    return das_mixed(Y, f.Gt, f.Gr, f.Ro, f.dt, f.delay, f.cp, "tfm", "ignore", "cuda", storage)


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_batch_matches_oracle(storage):
    """Every frame of one persistent launch against the reference's FP64 image
    of the same stored samples (1e-6 of max|Im|: a wrong index moves a pixel by
    O(1)), and against the one-frame kernel."""
    from dream_b200.batch import DASBatch
    frames = _frames(storage=storage)
    b = DASBatch(frames, storage=storage)
    assert b.items > 0 and b.grid > 0
    b.run()
    torch.cuda.synchronize()
    for i, f in enumerate(frames):
        ref = _expected(f, storage)
        got = f.Im.cpu().numpy().astype(np.float64)
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= 1e-6 * scale, f"frame {i}"
        assert float((f.Im - _single(f, storage)).abs().max()) <= 1e-6 * scale, f"frame {i}"


def test_batch_graph_replay_and_new_data():
    from dream_b200.batch import DASBatch
    frames = _frames(n=5, seed=12)
    b = DASBatch(frames)
    g = b.capture()
    for f in frames:
        f.Im.zero_()
    g.replay()
    torch.cuda.synchronize()
    first = [f.Im.clone() for f in frames]
    for f, r in zip(frames, first):
        ref = _expected(f, "f32")
        assert np.abs(r.cpu().numpy().astype(np.float64) - ref).max() <= 1e-6 * np.abs(ref).max()
    # new A-scans in the same buffers: the replay reads them
    for f in frames:
        f.Y.mul_(-2.0)
    g.replay()
    torch.cuda.synchronize()
    for f, r in zip(frames, first):
        assert torch.allclose(f.Im, -2.0 * r, rtol=1e-5, atol=1e-5 * float(r.abs().max()))


def test_autotune_cache_roundtrip():
    from dream_b200 import autotune
    f = _frames(n=1, seed=13)[0]
    a = autotune.tune(f.Y, f.Gt, f.Gr, f.Ro, f.dt, f.delay, f.cp, "tfm", "f32", nthr=128)
    assert a["tile"][0] * a["tile"][1] == 128 and a["jc"] in (8, 16)
    b = autotune.tune(f.Y, f.Gt, f.Gr, f.Ro, f.dt, f.delay, f.cp, "tfm", "f32", nthr=128)
    assert a == b
