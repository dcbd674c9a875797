"""The frame front-end and the streamed sequence on the GPU (ofc_to_gray, ofc_track_stream).

to_gray must equal the oracle's restatement of the CLI's arithmetic bit for bit (the oracle is pinned to the
reference's io.to_gray / io.downscale in test_oracle.py::test_to_gray). A streamed sequence must equal the array entry
points (ofc_track_sequence, ofc_track_sequence_hybrid, pinned to the reference's track_sequence in
test_gpu_sequence.py and test_gpu_hybrid.py) bit for bit: the same frames give the same results whether they come
from arrays or from a source through page-locked slots and the GPU's conversion."""
import threading

import numpy as np
import pytest
from conftest import golden

from optflow_b200 import Config, track_pair, track_sequence
from optflow_b200.stream import to_gray, track_stream

pytestmark = pytest.mark.gpu

FIELDS = ("ux", "uy", "conf", "raw_ux", "raw_uy", "valid")
STRAIN = ("Exx", "Eyy", "Exy", "gmax", "vol")


def same(a, b, label):
    for q in FIELDS:
        np.testing.assert_array_equal(getattr(a, q), getattr(b, q), err_msg=f"{label}: {q}")
    for q in STRAIN:
        np.testing.assert_array_equal(a.strain[q], b.strain[q], err_msg=f"{label}: {q}")
    for q in ("reference", "mean_conf", "n_fb_max", "fallback_frac", "fb_gate_rejected", "reacquired"):
        assert a.timing.get(q) == b.timing.get(q), (label, q)
    if a.fb is not None or b.fb is not None:
        np.testing.assert_array_equal(a.fb, b.fb, err_msg=f"{label}: fb")


def test_to_gray_matches_oracle(oracle):
    g = golden("frames")
    for name in ("gray8", "rgb24", "rgba32", "gray16", "rgb48", "f32"):
        for s in (1, 2, 3):
            want, _ = oracle.to_gray(g[f"{name}_in"], name, s)
            np.testing.assert_array_equal(to_gray(g[f"{name}_in"], s), want, err_msg=f"{name} scale {s}")
    with pytest.raises(ValueError, match="scale must be >= 1"):
        to_gray(g["gray8_in"], 0)


def test_stream_chain_equals_the_array_entry():
    gs = golden("seq")
    fr, roi = list(gs["frames"]), gs["roi"].astype(bool)
    for cfg in (Config(), Config(ref_update_conf=0.995)):
        want = dict(track_sequence(fr, cfg, mask=roi))
        got = dict(track_stream(iter(fr), cfg, mask=roi))
        assert sorted(got) == sorted(want) == list(range(1, len(fr)))
        for k in want:
            same(got[k], want[k], f"chain frame {k}")


def test_stream_hybrid_equals_the_array_entry():
    g = golden("hybrid")
    fr, roi = list(g["r_frames"]), g["r_roi"].astype(bool)
    cfg = Config(seq_mode="hybrid", fb_max=3, ref_update_conf=0.9)
    want = dict(track_sequence(fr, cfg, mask=roi))
    got = dict(track_stream(fr, cfg, mask=roi))
    assert sorted(got) == sorted(want)
    for k in want:
        same(got[k], want[k], f"hybrid frame {k}")


def test_stream_converts_rgb24_and_downscales_on_the_gpu(oracle):
    """rgb24 frames at twice the size (what ffmpeg hands the CLI for a video, with --scale 2): the stream's results
    equal the array entry's on the oracle's grey, downscaled frames."""
    gs = golden("seq")
    rng = np.random.default_rng(5)
    rgb = []
    for f in gs["frames"]:
        big = np.kron(f.astype(np.float64), np.ones((2, 2)))
        px = np.clip(np.rint(255 * big[..., None] + rng.normal(0, 2, big.shape + (3,))), 0, 255).astype(np.uint8)
        rgb.append(px)
    grey = [oracle.to_gray(p, "rgb24", 2)[0] for p in rgb]
    want = dict(track_sequence(grey, Config()))
    got = dict(track_stream(rgb, Config(), scale=2))
    for k in want:
        same(got[k], want[k], f"rgb24 frame {k}")


def test_stream_delivers_results_before_the_source_ends():
    """The engine reads one frame ahead: the first result arrives while most of a long source is still unread."""
    g = golden("hybrid")
    fr = list(g["f_frames"])  # 8 frames
    pulled = []

    def source():
        for f in fr:
            pulled.append(1)
            yield f

    seen = []
    for k, _ in track_stream(source(), Config()):
        seen.append((k, len(pulled)))
    assert [k for k, _ in seen] == list(range(1, len(fr)))
    assert seen[0][1] < len(fr), seen


def test_stream_errors_and_early_stop():
    gs = golden("seq")
    fr = list(gs["frames"])

    def broken():
        yield fr[0]
        yield fr[1]
        raise RuntimeError("decoder failed")

    with pytest.raises(RuntimeError, match="decoder failed"):
        list(track_stream(broken(), Config()))
    with pytest.raises(ValueError, match="frame 2 has shape"):
        list(track_stream([fr[0], fr[1], fr[2][:64]], Config()))
    with pytest.raises(ValueError, match="no frames"):
        next(track_stream([], Config()))
    # a consumer that stops after the first result: the run ends, the engine stays usable
    gen = track_stream(fr, Config())
    k, r = next(gen)
    gen.close()
    assert k == 1 and not any(t.name == "ofc_track_stream" for t in threading.enumerate())
    p = track_pair(fr[0], fr[1], Config(), mask=gs["roi"].astype(bool))
    assert np.isfinite(p.ux).any()
    assert list(track_stream(fr[:1], Config())) == []


def test_iter_frames_matches_the_reference():
    """iter_frames (GPU grey levels, downscale and window means) against the reference's io.iter_frames on the same
    frames (tests/golden/iter.npz): without averaging within float32 rounding; with averaging, the plain and the
    dense-aligned edge windows and the affine-aligned ones within 2e-3 away from the border (the reference warps with
    scipy's map_coordinates, the CLI and the engine with the B-spline of interp::warp; test_gpu_tavg.py)."""
    from optflow_b200.stream import iter_frames
    g = golden("iter")
    fr = list(g["frames"])
    mask = g["mask"].astype(bool)
    cfg = Config(max_disp=8.0)
    inner = (slice(20, -20), slice(20, -20))
    plain = list(iter_frames(iter(fr), start=2, stop=9, step=3, scale=2))
    assert len(plain) == len(g["plain"])
    for a, b in zip(plain, g["plain"]):
        assert np.abs(a - b).max() < 1e-6
    for name, kw in (("edge", dict(start=1, step=3, scale=2, tavg=2, cfg=cfg)),
                     ("aligned", dict(start=0, stop=7, step=2, scale=2, tavg=1, align=True, cfg=cfg,
                                      mask_fn=lambda shape: mask))):
        got = list(iter_frames(iter(fr), **kw))
        assert len(got) == len(g[name]), name
        for k, (a, b) in enumerate(zip(got, g[name])):
            assert np.abs(a[inner] - b[inner]).max() < 2e-3, (name, k, np.abs(a[inner] - b[inner]).max())
    with pytest.raises(ValueError, match="step must be >= 1"):
        next(iter_frames(iter(fr), step=0))
    # the averaged frames feed the streamed tracking as any frames do
    res = dict(track_stream(iter_frames(iter(fr), start=1, step=3, scale=2, tavg=2, cfg=cfg), Config()))
    assert sorted(res) == [1, 2] and all(np.isfinite(r.ux).any() for r in res.values())


@pytest.mark.parametrize("kw", [dict(start=1, step=3, tavg=2), dict(start=0, stop=7, step=2, tavg=1, align=True),
                                dict(start=2, stop=9, step=3), dict(start=0, step=2, tavg=1, hybrid=True)])
def test_stream_sampling_and_tavg_equal_iter_frames(kw):
    """The sampled and averaged frames made on the device inside the streamed driver (a ring of downscaled frames,
    window means, the edge windows aligned with the dense model, or every window with the affine model inside a
    mask) give the results of iter_frames' frames (pinned to the reference's io.iter_frames) through the array
    entry, bit for bit."""
    from optflow_b200.stream import iter_frames
    g = golden("iter")
    fr = list(g["frames"])
    mask = g["mask"].astype(bool)
    kw = dict(kw)
    cfg = Config(max_disp=8.0, seq_mode="hybrid" if kw.pop("hybrid", False) else "chain")
    mask_fn = (lambda shape: mask) if kw.get("align") else None
    frames = list(iter_frames(iter(fr), scale=2, cfg=cfg, mask_fn=mask_fn, **kw))
    want = dict(track_sequence(frames, cfg))
    got = dict(track_stream(iter(fr), cfg, scale=2, align_mask=mask if kw.get("align") else None, **kw))
    assert sorted(got) == sorted(want) == list(range(1, len(frames)))
    for k in want:
        same(got[k], want[k], f"{kw} frame {k}")
    with pytest.raises(ValueError, match="step must be >= 1"):
        next(track_stream(iter(fr), cfg, step=0))
