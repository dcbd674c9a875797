"""Pins the CPU oracle (oracle/oracle.cpp) before it is trusted as the checker of the CUDA engine.

Two anchors: the golden vectors in tests/golden (written by the reference's Python specification itself,
tests/golden/make_golden.py), checked to float32 storage precision; and, where the reference checkout is
present, the reference's own parity fixtures (rust/crates/optflow-core/tests/fixtures, written by
python/bench/make_parity_fixtures.py) with the tolerances of the reference's Rust parity tests.
"""
import os

import numpy as np
import pytest
from conftest import golden, ref_fixture, ref_meta, rms

from optflow_b200.config import Config


def close(a, b, tol):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    assert a.shape == b.shape
    assert np.array_equal(np.isnan(a), np.isnan(b)), "NaN patterns differ"
    m = np.isfinite(a)
    err = np.abs(a[m] - b[m]) / np.maximum(1.0, np.abs(b[m]))
    assert err.size == 0 or err.max() <= tol, f"max rel err {err.max():.3g} > {tol}"


# ---------------------------------------------------------------- golden vectors (float32-stored)
def test_fft_matches_numpy(oracle):
    rng = np.random.default_rng(0)
    for h, w in [(1, 5), (7, 12), (96, 160), (64, 64), (30, 151), (33, 121), (2, 2)]:
        a = rng.standard_normal((h, w)) + 1j * rng.standard_normal((h, w))
        for inv in (False, True):
            ref = np.fft.ifft2(a) if inv else np.fft.fft2(a)
            got = oracle.fft2(a, inv)
            assert np.abs(got - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())


def test_interp(oracle):
    g = golden("interp")
    img = g["img"].astype(np.float64)
    close(oracle.bspline_coeffs(img), g["coeffs"], 2e-6)
    c = oracle.bspline_coeffs(img)
    close(oracle.sample(c, g["x"].astype(np.float64), g["y"].astype(np.float64)), g["sample"], 2e-6)
    close(oracle.gauss_blur(img, 4.0), g["blur4"], 2e-6)
    close(oracle.gauss_blur(img, 1.0), g["blur1"], 2e-6)
    h, w = img.shape
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    warped = oracle.sample(c, xx + g["warp_ux"].astype(np.float32).astype(np.float64),
                           yy + g["warp_uy"].astype(np.float32).astype(np.float64))
    close(warped, g["warp"], 2e-6)


def test_edt_and_feature_transform(oracle):
    g = golden("edt")
    for s, d, idx in zip(g["src"], g["dist"], g["idx"]):
        dist, (iy, ix) = oracle.edt(~s.astype(bool), return_indices=True)
        np.testing.assert_array_equal(dist.astype(np.float32), d)
        np.testing.assert_array_equal(iy * s.shape[1] + ix, idx)


def test_gabor_reference_phase(oracle):
    g = golden("gabor")
    ref = oracle.reference_phase(g["img"].astype(np.float64), Config())
    scale = np.abs(g["r_re"] + 1j * g["r_im"]).max()
    for k, (r, gx, gy, amp) in enumerate(ref):
        assert np.abs(r.real - g["r_re"][k]).max() <= 1e-6 * scale
        assert np.abs(r.imag - g["r_im"][k]).max() <= 1e-6 * scale
        # the phase gradient divides by |r|^2 + 1e-12: compare where the response is not negligible
        m = np.abs(r) > 1e-4 * scale
        assert np.abs(gx - g["gx"][k])[m].max() <= 1e-4
        assert np.abs(gy - g["gy"][k])[m].max() <= 1e-4
        close(amp, g["amp"][k], 2e-6)


def test_strain(oracle):
    g = golden("strain")
    grads = oracle.displacement_gradient(g["ux"].astype(np.float64), g["uy"].astype(np.float64), 15)
    for got, k in zip(grads, ("dudx", "dudy", "dvdx", "dvdy")):
        close(got, g[k], 1e-6)
    _, _, st = oracle.finish(np.zeros((4, 4)), np.zeros((4, 4)), np.ones((4, 4)), Config(edge_guard=0.0))
    assert st["Exx"].shape == (4, 4)


def test_poc(oracle):
    g = golden("poc")
    a, b = g["a"].astype(np.float64), g["b"].astype(np.float64)
    dx, dy, pk = oracle.poc_shift(a[40:104, 50:114], b[40:104, 70:134])
    np.testing.assert_allclose([dx, dy, pk], g["shift"], atol=1e-9)
    assert oracle.n_levels(32.0, 64, a.shape) == int(g["n_levels"][0])
    r = oracle.coarse_flow(a, b, Config())
    np.testing.assert_array_equal(r["xs"], g["xs"])
    np.testing.assert_array_equal(r["ys"], g["ys"])
    for k in ("ux", "uy", "peak"):
        close(r[k], g[k], 2e-6)
    init = (g["init_ux"].astype(np.float64), g["init_uy"].astype(np.float64))
    r = oracle.coarse_flow(a, b, Config(), init_dense=init)
    close(r["ux"], g["iux"], 2e-6)
    close(r["uy"], g["iuy"], 2e-6)
    close(r["peak"], g["ipeak"], 2e-6)
    r = oracle.coarse_flow(a, np.full(a.shape, 0.5), Config(), init_dense=init)
    assert (r["peak"] == 0).all()
    close(r["ux"], g["fux"], 2e-6)
    close(r["uy"], g["fuy"], 2e-6)


@pytest.mark.parametrize("order", [1, 2])
def test_refine(oracle, order):
    g = golden("refine")
    f = oracle.refine(g["a"], g["b"], g["init_ux"], g["init_uy"], Config(shape_order=order))
    for k in ("ux", "uy", "conf", "resid"):
        close(f[k], g[f"o{order}_{k}"], 2e-6)


def test_refine_stripe_and_border(oracle):
    g = golden("stripe")
    f = oracle.refine(g["a"], g["b"], g["init_ux"], g["init_uy"], Config())
    close(f["ux"], g["ux"], 2e-6)
    close(f["conf"], g["conf"], 2e-6)
    assert f["conf"].max() < Config().conf_min
    g = golden("border")
    f = oracle.refine(g["a"], g["b"], g["init_ux"], g["init_uy"], Config(edge_guard=0.0))
    for k in ("ux", "uy", "conf"):
        close(f[k], g[k], 2e-6)


@pytest.mark.parametrize("name", ["pair_roi", "pair_affsin", "pair_init"])
def test_track_pair(oracle, name):
    g = golden(name)
    init = (g["init_ux"], g["init_uy"]) if "init_ux" in g else None
    r = oracle.track_pair(g["a"], g["b"], Config(), mask=g.get("roi"), init=init)
    for k in ("ux", "uy", "conf", "raw_ux", "raw_uy", "Exx", "Eyy", "Exy", "gmax", "vol"):
        close(r[k], g[k], 5e-6)


# ---------------------------------------------------------------- the reference's own fixtures
def _meta():
    return ref_meta()


def test_tavg(oracle):
    """The temporal-averaging restatement against the reference's tavg.py (tests/golden/tavg.npz): aligned frames
    agree away from the border (the reference warps with scipy's map_coordinates, the CLI with the B-spline of
    interp::warp), the plain mean exactly; the mask keeps the motion of the masked part only."""
    g = golden("tavg")
    cfg = Config(max_disp=8.0)
    fr = [f.astype(np.float64) for f in g["frames"]]
    m = (slice(20, -20), slice(20, -20))
    for got, want in ((oracle.align_to(fr[2], fr[0], cfg), g["aff0"]), (oracle.align_to(fr[2], fr[4], cfg), g["aff4"]),
                      (oracle.align_to(fr[0], g["split"], cfg, model="dense"), g["dense"]),
                      (oracle.align_to(g["m_static"], g["m_half"], cfg, mask=g["mask"].astype(bool)), g["masked"]),
                      (oracle.align_to(g["m_static"], g["m_half"], cfg), g["unmasked"]),
                      (oracle.average_window(fr, 2, align=True, cfg=cfg), g["aligned"])):
        assert np.abs(got[m] - want[m]).max() < 1e-6
    np.testing.assert_array_equal(oracle.average_window(fr, 2), g["plain"])
    assert oracle.align_to(np.full((128, 128), 0.5), np.full((128, 128), 0.5), cfg) is None


def test_ref_fixture_interp(oracle):
    img = ref_fixture("interp_img").astype(np.float64)
    x, y = ref_fixture("interp_x"), ref_fixture("interp_y")
    got = oracle.sample(oracle.bspline_coeffs(img), x, y)
    assert np.sqrt(np.mean((got - ref_fixture("interp_sample")) ** 2)) < 1e-5  # parity_interp.rs:46
    for s in (1, 2, 4):
        assert np.abs(oracle.gauss_blur(img, float(s)) - ref_fixture(f"interp_blur_{s}")).max() < 1e-6


def test_ref_fixture_gabor(oracle):
    img = ref_fixture("gabor_img").astype(np.float64)
    ref = oracle.reference_phase(img, Config())
    re, im = ref_fixture("gabor_r_re"), ref_fixture("gabor_r_im")
    scale = np.abs(re + 1j * im).max()
    for k, (r, gx, gy, _) in enumerate(ref):
        assert np.abs(r - (re[k] + 1j * im[k])).max() / scale < 1e-4  # parity_gabor.rs:68
        m = np.abs(r) > 1e-3 * scale
        assert np.abs(gx - ref_fixture("gabor_gx")[k])[m].max() < 1e-3  # parity_gabor.rs:69


def test_ref_fixture_poc(oracle):
    meta = _meta()
    a, b = ref_fixture("poc_a").astype(np.float64), ref_fixture("poc_b").astype(np.float64)
    y0, y1, x0, x1 = meta["poc_shift"]["window"]
    dx, dy, pk = oracle.poc_shift(a[y0:y1, x0:x1], b[y0:y1, x0:x1])
    assert abs(dx - meta["poc_shift"]["dx"]) < 1e-3 and abs(dy - meta["poc_shift"]["dy"]) < 1e-3
    r = oracle.coarse_flow(a, b, Config())
    for k in ("ux", "uy"):  # parity_poc.rs:50-51
        d = r[k] - ref_fixture(f"poc_grid_{k}")
        assert np.sqrt(np.mean(d ** 2)) < 1e-3 and np.abs(d).max() < 1e-3
    for h, w, lw in meta["level_window"]:
        assert oracle.level_window((h, w), 64) == (None if lw is None else tuple(lw))
    for d, h, w, L in meta["n_levels"]:
        assert oracle.n_levels(d, 64, (h, w)) == L
    sa, sb = ref_fixture("poc_strip_a").astype(np.float64), ref_fixture("poc_strip_b").astype(np.float64)
    r = oracle.coarse_flow(sa, sb, Config(max_disp=100))
    assert np.sqrt(np.mean((r["ux"] - ref_fixture("poc_strip_ux")) ** 2)) < 1e-3


@pytest.mark.parametrize("order", [1, 2])
def test_ref_fixture_refine(oracle, order):
    a, b = ref_fixture("refine_a"), ref_fixture("refine_b")
    f = oracle.refine(a, b, ref_fixture("refine_init_ux"), ref_fixture("refine_init_uy"), Config(shape_order=order))
    for k in ("ux", "uy", "conf", "resid"):  # parity_refine.rs:86-89
        assert rms(f[k], ref_fixture(f"refine_o{order}_{k}")) < 1e-3


def test_ref_fixture_strain_and_edt(oracle):
    grads = oracle.displacement_gradient(ref_fixture("strain_ux"), ref_fixture("strain_uy"), 15)
    for got, k in zip(grads, ("dudx", "dudy", "dvdx", "dvdy")):
        want = ref_fixture(f"strain_{k}")
        assert np.array_equal(np.isnan(got), np.isnan(want))
        assert np.nanmax(np.abs(got - want)) < 2e-7 * 10  # parity_strain.rs:12 (f32-stored inputs)
    valid = ref_fixture("edt_valid") > 0.5
    np.testing.assert_allclose(oracle.edt(valid), ref_fixture("edt_dist"), rtol=1e-6)
    for src, idx in zip(ref_fixture("edt_ft_src") > 0.5, ref_fixture("edt_ft_idx")):
        _, (iy, ix) = oracle.edt(~src, return_indices=True)
        np.testing.assert_array_equal(iy * src.shape[1] + ix, idx.astype(np.int64))


def test_ref_fixture_pair(oracle):
    a, b = ref_fixture("pair_a"), ref_fixture("pair_b")
    roi = ref_fixture("pair_roi") > 0.5
    r = oracle.track_pair(a, b, Config(), mask=roi)
    ux = ref_fixture("pair_ux")
    assert np.array_equal(np.isfinite(r["ux"]), np.isfinite(ux))  # parity_track.rs
    assert rms(r["ux"], ux) < 1e-3 and rms(r["uy"], ref_fixture("pair_uy")) < 1e-3
    assert rms(r["conf"], ref_fixture("pair_conf")) < 1e-3
    assert rms(r["Exx"], ref_fixture("pair_Exx")) < 1e-5 and rms(r["gmax"], ref_fixture("pair_gmax")) < 1e-5


def test_local_affine_agreement(oracle):
    """The hybrid gate's restatement against the reference's _local_affine_agreement (tests/golden/hybrid.npz): the
    plane with a hole at every radius, shift, support and tolerance of the golden cases, and the noisy field with a
    displacement step at radius 6.5 (rounded to 6, ties to even): ok and n exactly."""
    g = golden("hybrid")
    ux, uy, sup = g["laa_plane_ux"], g["laa_plane_uy"], g["laa_plane_support"].astype(bool)
    for c, (dx, radius, ms, tol) in enumerate(g["laa_plane_cases"]):
        ok, n = oracle.local_affine_agreement(ux, uy, sup, g["laa_plane_px"] + dx, g["laa_plane_py"], radius, ms, tol)
        np.testing.assert_array_equal(ok, g[f"laa_plane_ok{c}"].astype(bool), err_msg=f"case {c}")
        np.testing.assert_array_equal(n, g[f"laa_plane_n{c}"], err_msg=f"case {c}")
    sup = g["laa_step_support"].astype(bool)
    ok, n = oracle.local_affine_agreement(np.where(sup, g["laa_step_ux"], np.nan), np.where(sup, g["laa_step_uy"], np.nan),
                                          sup, g["laa_step_tx"], g["laa_step_ty"], 6.5, 20, 0.5)
    np.testing.assert_array_equal(ok, g["laa_step_ok"].astype(bool))
    np.testing.assert_array_equal(n, g["laa_step_n"])


def test_to_gray(oracle):
    """The frame front-end's restatement against the reference's io.to_gray / io.downscale (tests/golden/frames.npz):
    the grey levels exactly, the downscales within 1e-15 (numpy's mean sums in another order than the CLI), and the
    CLI's own known answers (io.rs:675-698)."""
    g = golden("frames")
    for name in ("gray8", "rgb24", "rgba32", "gray16", "rgb48", "f32"):
        out, grey = oracle.to_gray(g[f"{name}_in"], name)
        np.testing.assert_array_equal(grey, g[f"{name}_gray"], err_msg=name)
        np.testing.assert_array_equal(out, g[f"{name}_gray"].astype(np.float32), err_msg=name)
        for s in (2, 3):
            out, _ = oracle.to_gray(g[f"{name}_in"], name, s)
            want = g[f"{name}_down{s}"]
            assert out.shape == want.shape
            assert np.abs(out.astype(np.float64) - want).max() <= 1e-7 * np.abs(want).max(), (name, s)
    ramp = np.arange(16, dtype=np.float32).reshape(4, 4)
    np.testing.assert_array_equal(oracle.to_gray(ramp, "f32", 2)[0], [[2.5, 4.5], [10.5, 12.5]])
    blocks = np.array([[3 * y + x % 3 + 9 * (x // 3) for x in range(6)] for y in range(3)], np.float32)
    np.testing.assert_array_equal(oracle.to_gray(blocks, "f32", 3)[0], [[4.0, 13.0]])
    assert oracle.to_gray(np.ones((3, 5), np.float32), "f32", 2)[0].shape == (1, 2)


# ---------------------------------------------------------------- synthetic speckle (the benchmark's inputs)
def _synth_fields():
    from optflow_b200 import synth
    return {"none": None,
            "strain": synth.uniform_strain(0.01, -0.004, (40.0, 32.0), exy=0.003, t=(1.3, -0.7)),
            "sinaff": synth.Field(A=((1.01, 0.003), (0.003, 0.996)), c=(40.0, 32.0), t=(0.4, -0.25), amp=1.5,
                                  wavelength=32.0, s=(1.0, 1.0))}


def test_render_matches_the_reference_generator(oracle):
    """The oracle's restatement of synth.render against the reference's own renders (tests/golden/synth.npz, by
    make_golden_synth.py): the pattern draws exactly, the float64 images to 1e-12, the degraded 8-bit levels
    exactly. The GPU renderer is pinned to this restatement in the GPU tests."""
    from optflow_b200 import synth
    g = golden("synth")
    p = synth.make_pattern(64, 80, seed=3, rmin=1.5, rmax=2.5)
    for k in ("cx", "cy", "r", "a"):
        np.testing.assert_array_equal(getattr(p, k), g[k])
    for i, (name, f) in enumerate(_synth_fields().items()):
        img = oracle.render(p, 64, 80, f)
        assert np.abs(img - g[f"img_{name}"]).max() < 1e-12, name
        deg = synth.degrade(img, seed=10 + i, noise=0.01, bits=8)
        np.testing.assert_array_equal(np.round(deg.astype(np.float64) * 255), np.round(g[f"deg_{name}"] * 255))


def test_poc_integer_peaks_match_the_reference(oracle):
    """The integer POC peaks of every grid point of every pyramid level (the window offset plus the argmax of the
    last correlation surface) equal those of the reference's own coarse_flow on its POC fixtures
    (tests/golden/poc_peaks.npz, read from its poc_shift by make_golden_config2.py)."""
    g = golden("poc_peaks")
    a, b = ref_fixture("poc_a").astype(np.float64), ref_fixture("poc_b").astype(np.float64)
    sa, sb = ref_fixture("poc_strip_a").astype(np.float64), ref_fixture("poc_strip_b").astype(np.float64)
    for name, (x, y, cfg) in {"grid": (a, b, Config()), "strip": (sa, sb, Config(max_disp=100))}.items():
        levels = sorted(k for k in g if k.startswith(name + "_l"))
        for lev, key in enumerate(levels):
            np.testing.assert_array_equal(oracle.coarse_peaks(x, y, cfg, level=lev), g[key], err_msg=key)
        assert oracle.coarse_peaks(x, y, cfg, level=len(levels)) is None
