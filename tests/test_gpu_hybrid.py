"""seq_mode "hybrid" on the GPU (ofc_track_sequence_hybrid, ofc_local_affine_agreement) against the reference's own
hybrid mode (tests/golden/hybrid.npz, written by tests/golden/make_golden_hybrid.py from python/optflow_ref/track.py:
331-503).

Scripted legs (tests/hybrid_scripts.py, the scenarios of the reference's python/tests/test_hybrid.py) give every
decision of the state machine exactly: the fallback counters, validity and the reference index bit for bit, fields and
confidences within float32 rounding. Real frames (a pattern whose patch fades into another) go through the engine's
own legs and compare with the bars of compare_hybrid (the pair bars where the pixel classes agree)."""
import numpy as np
import pytest
from conftest import golden, rms
from test_gpu_parity import DISP_TOL, STRAIN_TOL

import hybrid_scripts as S
from optflow_b200 import Config, local_affine_agreement, track_sequence, track_sequence_hybrid

pytestmark = pytest.mark.gpu

TIMING = ("reference", "mean_conf", "n_fb_max", "fallback_frac", "fb_gate_rejected", "reacquired")


@pytest.fixture(scope="module")
def g():
    return golden("hybrid")


def test_local_affine_agreement_golden(g):
    ux, uy, sup = g["laa_plane_ux"], g["laa_plane_uy"], g["laa_plane_support"].astype(bool)
    for c, (dx, radius, ms, tol) in enumerate(g["laa_plane_cases"]):
        ok, n = local_affine_agreement(ux, uy, sup, g["laa_plane_px"] + dx, g["laa_plane_py"], radius, int(ms), tol)
        np.testing.assert_array_equal(ok, g[f"laa_plane_ok{c}"].astype(bool), err_msg=f"case {c}")
        np.testing.assert_array_equal(n, g[f"laa_plane_n{c}"], err_msg=f"case {c}")
    sup = g["laa_step_support"].astype(bool)
    ok, n = local_affine_agreement(np.where(sup, g["laa_step_ux"], np.nan), np.where(sup, g["laa_step_uy"], np.nan), sup,
                                   g["laa_step_tx"], g["laa_step_ty"], 6.5, 20, 0.5)
    np.testing.assert_array_equal(ok, g["laa_step_ok"].astype(bool))
    np.testing.assert_array_equal(n, g["laa_step_n"])


def _scripted(name, **over):
    n = S.SCENARIOS[name][0]
    calls = []

    def legs(i, j, init):
        calls.append((i, j, init is not None))
        return S.leg(name, i, j)

    out = dict(track_sequence_hybrid(S.frames(n), Config(**dict(S.config_keys(name), **over)),
                                     ref_update_conf=S.ruc_list(name), legs=legs))
    return out, calls


@pytest.mark.parametrize("name", sorted(S.SCENARIOS))
def test_scripted_scenarios_golden(g, name):
    out, _ = _scripted(name)
    for k, r in out.items():
        p = f"s_{name}_{k}_"
        np.testing.assert_array_equal(r.fb, g[p + "fb"], err_msg=f"{name} frame {k}: fb")
        np.testing.assert_array_equal(np.isfinite(r.ux), np.isfinite(g[p + "ux"]), err_msg=f"{name} frame {k}: valid")
        for q in ("ux", "uy", "conf", "raw_ux", "raw_uy"):
            np.testing.assert_allclose(getattr(r, q), g[p + q], rtol=0, atol=1e-5, equal_nan=True,
                                       err_msg=f"{name} frame {k}: {q}")
        want = dict(zip(TIMING, g[p + "timing"]))
        for q in ("reference", "n_fb_max"):
            assert r.timing[q] == int(want[q]), (name, k, q)
        for q in ("mean_conf", "fallback_frac", "fb_gate_rejected", "reacquired"):
            assert abs(r.timing[q] - want[q]) < 1e-6, (name, k, q, r.timing[q], want[q])


def test_scripted_fallback_reads_like_the_reference_tests():
    """Three of the reference's own assertions (python/tests/test_hybrid.py:108-121, 155-168, 270-283), on the
    engine: the counter expires at fb_max, a pixel in fallback when the reference moves stays unanchored, and a
    confident direct value 1 px off the carried one is not re-acquired."""
    out, calls = _scripted("expiry")
    P = S.PATCH
    for k, n in ((2, 1), (3, 2), (4, 3)):
        assert (out[k].fb[P] == n).all() and out[k].ux[40, 40] == pytest.approx(k)
        assert out[k].conf[40, 40] == pytest.approx(0.9 * (1 - n / 4))
    for k in (5, 6):
        assert np.isnan(out[k].ux[40, 40]) and np.isfinite(out[k].ux[70, 70]) and (out[k].fb[P] == 4).all()
    # frame 1 has no previous leg: no dense start; frames from 2 on start from the last direct leg
    assert calls[0] == (0, 1, False) and all(c[2] for c in calls if c[:2] == (0, 5))
    out, _ = _scripted("unanchored")
    assert out[4].timing["reference"] == 3 and (out[4].fb[P] == 2).all() and out[4].ux[40, 40] == pytest.approx(4.0)
    assert np.isnan(out[8].ux[40, 40]) and (out[8].fb[P] == 6).all()
    out, _ = _scripted("no_recover")
    assert (out[6].fb[30:50, 30:44] == 4).all() and out[6].ux[40, 40] == pytest.approx(6.0)
    assert (out[7].fb[30:50, 30:44] == 5).all() and np.isnan(out[7].ux[40, 40])
    off, _ = _scripted("no_recover_v2")
    assert (off[7].fb[30:50, 30:44] == 0).all() and off[7].ux[40, 40] == pytest.approx(8.0)


def compare_hybrid(r, want, label):
    """Parity of a hybrid frame with the reference's: the fallback counters on 99 % of the ROI; validity on 98 % of
    the image (a fallback pixel is valid by the spatial gate, not by its confidence, so its flips need not sit at
    conf_min); fields on the pixels valid in both, confidence and the unmasked field where both are direct-good
    (fb == 0) and the reference's confidence reaches conf_min; strain where no validity flip enters its window."""
    from scipy.ndimage import binary_dilation
    roi = want["roi"]
    same = r.fb == want["fb"]
    assert same[roi].mean() > 0.99, (label, same[roi].mean())
    vg, vw = np.isfinite(r.ux), np.isfinite(want["ux"])
    diff = vg != vw
    assert diff.mean() < 0.02, (label, diff.mean())
    both = vg & vw
    assert both.sum() > 0.9 * vw.sum(), label
    assert rms(r.ux, want["ux"], both) < DISP_TOL and rms(r.uy, want["uy"], both) < DISP_TOL, label
    direct = (r.fb == 0) & (want["fb"] == 0) & (want["conf"] >= Config().conf_min)
    assert rms(r.conf, want["conf"], direct) < DISP_TOL, label
    assert rms(r.raw_ux, want["raw_ux"], direct) < DISP_TOL and rms(r.raw_uy, want["raw_uy"], direct) < DISP_TOL, label
    h = Config().strain_win // 2
    calm = both & ~binary_dilation(diff, structure=np.ones((2 * h + 1, 2 * h + 1), bool))
    for k in ("Exx", "Eyy", "Exy", "gmax", "vol"):
        m = calm & np.isfinite(r.strain[k]) & np.isfinite(want[k])
        assert rms(r.strain[k], want[k], m) < STRAIN_TOL, (label, k)


@pytest.mark.parametrize("tag", ["a", "b"])
def test_real_frames_golden(g, tag):
    fr, roi = list(g["r_frames"]), g["r_roi"].astype(bool)
    cfg = Config(seq_mode="hybrid", fb_max=3, ref_update_conf=0.0 if tag == "a" else 0.9)
    seen = 0
    for k, r in track_sequence(fr, cfg, mask=roi):
        p = f"r{tag}{k}_"
        want = {q: g[p + q] for q in ("ux", "uy", "conf", "raw_ux", "raw_uy", "fb", "Exx", "Eyy", "Exy", "gmax",
                                      "vol")}
        want["roi"] = roi
        compare_hybrid(r, want, f"hybrid {tag} frame {k}")
        t = dict(zip(TIMING, g[p + "timing"]))
        assert r.timing["reference"] == int(t["reference"]) and r.timing["n_fb_max"] == int(t["n_fb_max"]), (tag, k)
        assert abs(r.timing["mean_conf"] - t["mean_conf"]) < 1e-3, (tag, k)
        for q in ("fallback_frac", "fb_gate_rejected", "reacquired"):
            assert abs(r.timing[q] - t[q]) < 0.01, (tag, k, q, r.timing[q], t[q])
        seen += 1
    assert seen == len(fr) - 1


@pytest.mark.parametrize("name,fb_max", [("A", 10), ("B", 2)])
def test_reference_fixtures(g, name, fb_max):
    """The reference's committed hybrid fixtures (a translation with a foreign block; the reference moves, pixels are
    carried, the gate rejects some, the direct leg re-acquires others) with the bars of its own Rust parity test
    (rust/crates/optflow-core/tests/parity_track.rs:550-629): reference and n_fb_max exactly, mean confidence within
    1e-4, the shares within 2e-3, fb equal on 99.9 % of the pixels, NaN agreement 99.5 %, rms ux and (A) conf
    below 1e-3."""
    fr = list(g["f_frames"])
    out = list(track_sequence(fr, Config(seq_mode="hybrid", ref_update_conf=0.8, fb_max=fb_max)))
    assert len(out) == len(fr) - 1
    for (k, r), t in zip(out, g[f"f_{name}_timing"]):
        t = dict(zip(TIMING, t))
        wx = g[f"f_{name}_ux"][k - 1]
        assert r.timing["reference"] == int(t["reference"]), (name, k)
        assert r.timing["n_fb_max"] == int(t["n_fb_max"]), (name, k)
        assert abs(r.timing["mean_conf"] - t["mean_conf"]) < 1e-4, (name, k)
        for q in ("fallback_frac", "fb_gate_rejected", "reacquired"):
            assert abs(r.timing[q] - t[q]) < 2e-3, (name, k, q, r.timing[q], t[q])
        assert (r.fb == g[f"f_{name}_fb"][k - 1]).mean() >= 0.999, (name, k)
        assert (np.isfinite(r.ux) == np.isfinite(wx)).mean() >= 0.995, (name, k)
        assert rms(r.ux, wx, np.isfinite(r.ux) & np.isfinite(wx)) < 1e-3, (name, k)
        if name == "A":
            assert rms(r.conf, g["f_A_conf"][k - 1]) < 1e-3, (name, k)


def test_all_good_hybrid_equals_chain():
    """Where every pixel stays direct-good (fb == 0), the hybrid output is the chain's bit for bit (the reference's
    test_all_good_real_images_hybrid_is_bit_identical_to_chain, python/tests/test_hybrid.py:84-95)."""
    gs = golden("seq")
    fr, roi = list(gs["frames"]), gs["roi"].astype(bool)
    chain = dict(track_sequence(fr, Config(), mask=roi))
    hyb = dict(track_sequence(fr, Config(seq_mode="hybrid"), mask=roi))
    for k in chain:
        good = hyb[k].fb == 0
        assert good[roi].mean() > 0.85  # the rest: the ROI's border strip, where the direct leg's confidence is 0
        for q in ("raw_ux", "raw_uy", "conf"):
            np.testing.assert_array_equal(getattr(hyb[k], q)[good], getattr(chain[k], q)[good], err_msg=q)
        v = good & np.isfinite(chain[k].ux)
        np.testing.assert_array_equal(hyb[k].ux[v], chain[k].ux[v])


def test_hybrid_arguments():
    fr = S.frames(3)
    with pytest.raises(ValueError, match="fb_max must be >= 0"):
        next(track_sequence(fr, Config(seq_mode="hybrid", fb_max=-1)))
    with pytest.raises(ValueError, match="fb_tol finite and positive"):
        next(track_sequence(fr, Config(seq_mode="hybrid", fb_tol=0.0)))
    with pytest.raises(ValueError, match="one value per frame"):
        next(track_sequence_hybrid(fr, Config(seq_mode="hybrid"), ref_update_conf=[0.5]))

    def broken(i, j, init):
        raise RuntimeError(f"no leg {i} -> {j}")

    with pytest.raises(RuntimeError, match="no leg 0 -> 1"):
        next(track_sequence_hybrid(fr, Config(seq_mode="hybrid"), legs=broken))
    assert list(track_sequence(fr[:1], Config(seq_mode="hybrid"))) == []
