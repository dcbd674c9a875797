"""The CUDA engine against the reference, through the C ABI: golden vectors written by the reference itself
(tests/golden) and the CPU oracle on seeded inputs.

Bars (the reference's own parity tests and the pair path's contract): ux, uy, conf, resid RMS < 1e-3
(rust/crates/optflow-core/tests/parity_refine.rs:86-89); POC grid within 1e-3 px (parity_poc.rs:50-51);
strain RMS < 1e-5 (parity_track.rs:70-72); validity masks identical except at pixels whose confidence is
within a small distance of conf_min or whose guard decision follows from such a pixel.
"""
import numpy as np
import pytest
from conftest import golden, rms

from optflow_b200 import Config, coarse_flow, displacement_gradient, refine, track_pair

pytestmark = pytest.mark.gpu

DISP_TOL = 1e-3
STRAIN_TOL = 1e-5


@pytest.mark.parametrize("order", [1, 2])
def test_refine_golden(order):
    g = golden("refine")
    f = refine(g["a"], g["b"], g["init_ux"], g["init_uy"], Config(shape_order=order))
    for k in ("ux", "uy", "conf", "resid"):
        assert rms(getattr(f, k), g[f"o{order}_{k}"]) < DISP_TOL, k
    assert np.abs(f.ux - g[f"o{order}_ux"]).max() < 1e-2


def test_refine_stripe_is_degenerate():
    g = golden("stripe")
    f = refine(g["a"], g["b"], g["init_ux"], g["init_uy"], Config())
    assert f.conf.max() < Config().conf_min
    assert np.isfinite(f.ux).all() and np.isfinite(f.uy).all()
    assert rms(f.ux, g["ux"]) < DISP_TOL and rms(f.uy, g["uy"]) < DISP_TOL


def test_refine_border_guard_off():
    g = golden("border")
    f = refine(g["a"], g["b"], g["init_ux"], g["init_uy"], Config(edge_guard=0.0))
    assert (f.conf[:, :2] == 0).all() and (f.conf[-2:, :] == 0).all()
    np.testing.assert_array_equal(f.conf == 0, g["conf"] == 0)
    for k in ("ux", "uy", "conf"):
        assert rms(getattr(f, k), g[k]) < DISP_TOL


def test_coarse_flow_golden():
    g = golden("poc")
    r = coarse_flow(g["a"], g["b"], Config())
    np.testing.assert_array_equal(r.xs, g["xs"])
    np.testing.assert_array_equal(r.ys, g["ys"])
    for k in ("ux", "uy", "peak"):
        assert np.abs(getattr(r, k) - g[k]).max() < DISP_TOL, k
    r = coarse_flow(g["a"], g["b"], Config(), init_dense=(g["init_ux"], g["init_uy"]))
    assert np.abs(r.ux - g["iux"]).max() < DISP_TOL and np.abs(r.uy - g["iuy"]).max() < DISP_TOL
    assert np.abs(r.peak - g["ipeak"]).max() < DISP_TOL
    r = coarse_flow(g["a"], np.full(g["a"].shape, 0.5, np.float32), Config(), init_dense=(g["init_ux"], g["init_uy"]))
    assert (r.peak == 0).all()
    assert np.abs(r.ux - g["fux"]).max() < 1e-5 and np.abs(r.uy - g["fuy"]).max() < 1e-5


def test_strain_golden():
    g = golden("strain")
    got = displacement_gradient(g["ux"], g["uy"], 15)
    for a, k in zip(got, ("dudx", "dudy", "dvdx", "dvdy")):
        np.testing.assert_array_equal(np.isnan(a), np.isnan(g[k]))
        assert np.nanmax(np.abs(a - g[k])) < 1e-6


def compare_pair(r, want, label, conf_band=0.02, max_bars=True):
    """Parity of a track_pair Result with the reference's outputs (want: dict of arrays)."""
    valid_g = np.isfinite(r.ux)
    valid_w = np.isfinite(want["ux"])
    both = valid_g & valid_w
    # validity: every disagreement must sit where the confidence is within conf_band of conf_min, or within
    # the guard distance of such a pixel (a flipped low pixel moves the guard band around it)
    cmin = Config().conf_min
    near = np.abs(np.asarray(want["conf"], np.float64) - cmin) < conf_band
    diff = valid_g != valid_w
    if diff.any():
        from scipy.ndimage import binary_dilation
        zone = binary_dilation(near, iterations=int(np.ceil(Config().edge_guard_px())) + 1)
        assert (diff & ~zone).sum() == 0, f"{label}: {int((diff & ~zone).sum())} validity differences away from threshold"
    assert diff.mean() < 0.01, f"{label}: {diff.mean():.4f} of pixels change validity"
    assert both.sum() > 0.5 * valid_w.sum()
    assert rms(r.ux, want["ux"], both) < DISP_TOL, label
    assert rms(r.uy, want["uy"], both) < DISP_TOL, label
    dmax = {k: float(np.abs(np.asarray(getattr(r, k), np.float64)[both] - want[k][both]).max()) for k in ("ux", "uy")}
    smax = {}
    for k in ("Exx", "Eyy", "Exy", "gmax", "vol"):
        m = both & np.isfinite(r.strain[k]) & np.isfinite(want[k])
        smax[k] = float(np.abs(np.asarray(r.strain[k], np.float64)[m] - want[k][m]).max()) if m.any() else 0.0
    low_flip = (np.asarray(r.conf, np.float64) < cmin) != (np.asarray(want["conf"], np.float64) < cmin)
    band = float(np.abs(np.asarray(want["conf"], np.float64)[low_flip] - cmin).max()) if low_flip.any() else 0.0
    print(f"PAIRMAX {label} validity diffs {int(diff.sum())} low flips {int(low_flip.sum())} band {band:.2e} "
          f"field_max {dmax} strain_max {smax}", flush=True)
    if max_bars:
        # the pair contract in its own words: fields within 1e-3 px and strains within 1e-5 at every pixel (measured
        # on these pairs: at most 4.2e-6 px and 4.7e-7)
        assert max(dmax.values()) < DISP_TOL and max(smax.values()) < STRAIN_TOL, (label, dmax, smax)
    assert rms(r.conf, want["conf"]) < DISP_TOL, label
    # the unmasked field (the init of a sequence's next frame; not a CLI output) on the confident pixels
    trusted = np.asarray(want["conf"]) >= cmin
    assert rms(r.raw_ux, want["raw_ux"], trusted) < DISP_TOL and rms(r.raw_uy, want["raw_uy"], trusted) < DISP_TOL, label
    for k in ("Exx", "Eyy", "Exy", "gmax", "vol"):
        m = both & np.isfinite(r.strain[k]) & np.isfinite(want[k])
        assert rms(r.strain[k], want[k], m) < STRAIN_TOL, (label, k)


@pytest.mark.parametrize("name", ["pair_roi", "pair_affsin", "pair_init", "pair_seq256"])
def test_track_pair_golden(name):
    g = golden(name)
    init = (g["init_ux"], g["init_uy"]) if "init_ux" in g else None
    r = track_pair(g["a"], g["b"], Config(), mask=g.get("roi"), init=init)
    compare_pair(r, g, name)
    np.testing.assert_array_equal(r.valid, np.isfinite(r.ux))


def _synthetic_pair(n, seed, t=(2.3, -1.4), exx=0.01, noise=0.01):
    """A seeded speckle pair (Gaussian blobs, affine deformation) for the oracle comparisons."""
    rng = np.random.default_rng(seed)
    nb = int(0.6 * (n + 40) ** 2 / (np.pi * 4.0))
    cx, cy = rng.uniform(-20, n + 20, (2, nb))
    r = rng.uniform(1.5, 2.5, nb)
    a = rng.uniform(0.3, 1.0, nb) * rng.choice([-1.0, 1.0], nb)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)

    def render(X, Y):
        acc = np.zeros((n, n))
        for k in range(nb):
            x0, x1 = int(max(cx[k] - 12, 0)), int(min(cx[k] + 13, n))
            y0, y1 = int(max(cy[k] - 12, 0)), int(min(cy[k] + 13, n))
            if x0 >= x1 or y0 >= y1:
                continue
            dx = X[y0:y1, x0:x1] - cx[k]
            dy = Y[y0:y1, x0:x1] - cy[k]
            acc[y0:y1, x0:x1] += a[k] * np.exp(-(dx * dx + dy * dy) / (2 * r[k] ** 2))
        return 0.5 + 0.25 * np.tanh(acc)

    c = n / 2
    X = c + (xx - c - t[0]) / (1 + exx)
    Y = yy - t[1]
    i1 = render(xx, yy) + rng.normal(0, noise, (n, n))
    i2 = render(X, Y) + rng.normal(0, noise, (n, n))
    q = lambda im: (np.round(np.clip(im, 0, 1) * 255) / 255).astype(np.float32)
    return q(i1), q(i2)


@pytest.mark.parametrize("n,seed", [(192, 1), (256, 2)])
def test_track_pair_oracle(oracle, n, seed):
    a, b = _synthetic_pair(n, seed)
    roi = np.zeros((n, n), bool)
    roi[n // 10:n - n // 10, n // 8:n - n // 8] = True
    want = oracle.track_pair(a, b, Config(), mask=roi)
    r = track_pair(a, b, Config(), mask=roi)
    compare_pair(r, want, f"oracle{n}")


def test_track_pair_bluestein_sizes(oracle):
    """A pair whose padded sizes have prime factors above 31 (127 x 100 -> 191 x 164 = 191 x 4 * 41: every transform
    through Bluestein's chirp z-transform) against the oracle with the pair bars; a 960 x 540 frame (padded height
    604 = 4 * 151, the CLI's 1920 x 1080 video at --scale 2) passes check_window."""
    from optflow_b200.api import default_engine
    a, b = _synthetic_pair(192, 21)
    a, b = a[20:120, 30:157], b[20:120, 30:157]
    want = oracle.track_pair(a, b, Config())
    r = track_pair(a, b, Config())
    compare_pair(r, want, "bluestein 127x100")
    default_engine().check_window(960, 540, Config())


def test_refine_raw_window_shift(oracle):
    """refine_raw on a window of a larger pair (FineEngine::refine_raw with a shift) equals refine on the crop
    when the second image's window covers the displaced positions."""
    from optflow_b200 import refine_raw
    a, b = _synthetic_pair(192, 7, t=(1.2, 0.7), exx=0.0)
    x0, y0, w, h = 40, 32, 96, 112
    u = np.full((h, w), 1.2, np.float32)
    v = np.full((h, w), 0.7, np.float32)
    sx, sy = x0 - 16, y0 - 16
    i2 = b[sy:sy + h + 64, sx:sx + w + 64]
    got = refine_raw(a[y0:y0 + h, x0:x0 + w], i2, u, v, Config(), shift=(x0 - sx, y0 - sy))
    want = oracle.refine(a[y0:y0 + h, x0:x0 + w], b[y0:y0 + h, x0:x0 + w], u, v, Config())
    inner = (slice(20, -20), slice(20, -20))
    assert rms(got["ux"][inner], want["ux"][inner]) < 5e-3


def test_refine_batch_equals_refine_raw():
    """ofc_refine_batch (the tile loop's refine_raw calls in one call, copies on a second stream) gives each
    window's refine_raw result bit for bit, for windows of different sizes and shifts; a bad window is refused
    by index before any work."""
    from optflow_b200 import EngineError, refine_batch, refine_raw
    a, b = _synthetic_pair(192, 11, t=(0.9, -0.6), exx=0.004)
    wins = []
    for (x0, y0, w, h) in ((40, 32, 96, 112), (0, 0, 128, 96), (24, 40, 160, 128), (40, 32, 96, 112)):
        u = np.full((h, w), 0.9, np.float32)
        v = np.full((h, w), -0.6, np.float32)
        sx, sy = max(x0 - 16, 0), max(y0 - 16, 0)
        i2 = b[sy:sy + h + 32, sx:sx + w + 32]
        wins.append((a[y0:y0 + h, x0:x0 + w], i2, u, v, (x0 - sx, y0 - sy)))
    got = refine_batch(wins, Config())
    assert len(got) == len(wins)
    for k, (i1, i2, u, v, sh) in enumerate(wins):
        want = refine_raw(i1, i2, u, v, Config(), shift=sh)
        for q in ("ux", "uy", "energy", "resid"):
            assert np.array_equal(got[k][q], want[q], equal_nan=True), (k, q)
    assert refine_batch([], Config()) == []
    z = np.zeros((0, 0), np.float32)
    with pytest.raises(ValueError, match="window 1: empty"):
        refine_batch(wins[:1] + [(z, z, z, z, (0, 0))], Config())
    # padded height 4099, a prime: Bluestein's inner length 8232 leaves no room for the column pass in shared memory
    tall = np.zeros((4035, 45), np.float32)
    with pytest.raises(EngineError, match="window 2"):
        refine_batch(wins[:2] + [(tall, tall, tall, tall, (0, 0))], Config())


def test_track_pair_graph_replay_and_device_api():
    """The first call of a (size, configuration) runs eagerly and captures the pair as CUDA graphs; later calls
    replay them. Replays, a different size in between (which reallocates the pooled buffers and drops the
    graphs) and the device-resident entry point on a caller's stream all give the eager call's outputs."""
    import torch
    from optflow_b200 import Engine, track_pair_device
    a, b = _synthetic_pair(192, 11)
    roi = np.zeros(a.shape, bool)
    roi[10:-10, 12:-12] = True
    eng = Engine(0)
    try:
        first = track_pair(a, b, Config(), mask=roi, engine=eng)
        launches = eng.kernel_launches()
        again = track_pair(a, b, Config(), mask=roi, engine=eng)
        per_pair = eng.kernel_launches() - launches
        assert per_pair > 0
        big = _synthetic_pair(256, 12)
        track_pair(big[0], big[1], Config(), engine=eng)
        third = track_pair(a, b, Config(), mask=roi, engine=eng)
        fourth = track_pair(a, b, Config(), mask=roi, engine=eng)
        for r in (again, third, fourth):
            for k in ("ux", "uy", "conf", "raw_ux", "raw_uy", "valid"):
                np.testing.assert_array_equal(getattr(r, k), getattr(first, k), err_msg=k)
            for k in ("Exx", "Eyy", "Exy", "gmax", "vol"):
                np.testing.assert_array_equal(r.strain[k], first.strain[k], err_msg=k)
        # another pair of the same size between replays: each call downloads its own outputs (the host call
        # downloads some planes on a second stream while the pair's last stages run)
        c, d = _synthetic_pair(192, 13, t=(0.4, -1.1))
        other = track_pair(c, d, Config(), mask=roi, engine=eng)
        fifth = track_pair(a, b, Config(), mask=roi, engine=eng)
        eng2 = Engine(0)
        try:
            other_eager = track_pair(c, d, Config(), mask=roi, engine=eng2)
        finally:
            eng2.close()
        for k in ("ux", "uy", "conf", "raw_ux", "raw_uy", "valid"):
            np.testing.assert_array_equal(getattr(other, k), getattr(other_eager, k), err_msg=k)
            np.testing.assert_array_equal(getattr(fifth, k), getattr(first, k), err_msg=k)
        for k in ("Exx", "Eyy", "Exy", "gmax", "vol"):
            np.testing.assert_array_equal(other.strain[k], other_eager.strain[k], err_msg=k)
        assert not np.array_equal(other.raw_ux, first.raw_ux)
        st = torch.cuda.Stream()
        ta, tb, tr = (torch.from_numpy(x).cuda() for x in (a, b, roi))
        for _ in range(2):
            with torch.cuda.stream(st):
                out = track_pair_device(ta, tb, Config(), mask=tr, stream=st, engine=eng)
            st.synchronize()
            np.testing.assert_array_equal(out["ux"].cpu().numpy(), first.ux)
            np.testing.assert_array_equal(out["conf"].cpu().numpy(), first.conf)
            np.testing.assert_array_equal(out["valid"].cpu().numpy().astype(bool), first.valid)
            np.testing.assert_array_equal(out["exx"].cpu().numpy(), first.strain["Exx"])
    finally:
        eng.close()


def test_profile_mode_counts_replayed_kernels():
    """Profile mode (per-kernel device times, the reference's OPTFLOW_GPU_KERNELS) sees every launch of a
    replayed pair graph: the accumulation runs outer_iters x inner_iters times per pair."""
    import ctypes
    from optflow_b200 import Engine
    a, b = _synthetic_pair(192, 13)
    eng = Engine(0)
    try:
        eng.lib.ofc_set_profile(eng.handle, b"k_accumulate")
        for _ in range(3):
            track_pair(a, b, Config(), engine=eng)
        cap = 8
        names = ctypes.create_string_buffer(cap * 64)
        counts = (ctypes.c_uint64 * cap)()
        ms = (ctypes.c_double * cap)()
        n = eng.lib.ofc_profile_read(eng.handle, names, 64, counts, ms, cap)
        eng.lib.ofc_set_profile(eng.handle, None)
        got = {names.raw[i * 64:(i + 1) * 64].split(b"\0", 1)[0].decode(): (counts[i], ms[i]) for i in range(n)}
        cfg = Config()
        assert got["k_accumulate"][0] == 3 * cfg.outer_iters * cfg.inner_iters
        assert got["k_accumulate"][1] > 0
    finally:
        eng.close()


def test_busy_lane_refuses_instead_of_waiting():
    """A call beyond the engine's lanes is refused with OFC_ERR_BUSY (3) at once, like the Metal engine's
    per-lane try_lock (rust/crates/optflow-gpu/src/engine.rs:660-676); the lane is free again afterwards."""
    import threading
    from optflow_b200 import Engine, EngineError
    a, b = _synthetic_pair(512, 14)
    eng = Engine(0, lanes=1)
    try:
        track_pair(a, b, Config(), engine=eng)  # buffers and graphs exist: the next call is replay-only
        done = threading.Event()

        def work():
            while True:  # the main thread's probes can hold the lane for a moment: retry those refusals
                try:
                    track_pair(a, b, Config(), engine=eng)
                    break
                except EngineError as e:
                    if e.status != 3:
                        raise
            done.set()

        worker = threading.Thread(target=work)
        busy = 0
        worker.start()
        while not done.is_set() and worker.is_alive():
            try:
                eng.check_window(512, 512)
            except EngineError as e:
                assert e.status == 3 and "busy" in str(e)
                busy += 1
        worker.join()
        assert busy > 0
        eng.check_window(512, 512)
    finally:
        eng.close()
