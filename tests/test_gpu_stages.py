"""Each CUDA stage against the reference's intermediate arrays (through include/optflow_cuda_testing.h).

The expected values come from the committed golden vectors (written by the reference itself) and from the
CPU oracle, which tests/test_oracle.py pins to the reference.
"""
import numpy as np
import pytest
from conftest import golden

from optflow_b200.config import Config

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T():
    from optflow_b200 import testing
    return testing


# direct plans (radices up to 31; 320 ... 2112 on plans fixed at compile time), then lengths with a larger prime factor
# (Bluestein: 37, 41 * 4, 2 * 53, 151 * 4 = the padded height of a 960 x 540 frame (inner length 1216, on a fixed
# plan), the primes 191 and 1021, and 1999 = the largest inner length here, 4096)
BLUESTEIN = [37, 164, 106, 604, 191, 1021, 1999]


@pytest.mark.parametrize("L", [64, 128, 160, 192, 224, 320, 576, 832, 1024, 1088, 1152, 1600, 2112, 2*3*5*7*11, 3*17*19,
                               23*29, 31*8]
                         + BLUESTEIN)
def test_fft_lines_match_numpy(T, L):
    """Line transforms against numpy in float64: 2e-6 of the largest output for the direct plans, 1e-5 for
    Bluestein's (a float32 chirp, two transforms of the inner length and a product between them)."""
    rng = np.random.default_rng(L)
    a = (rng.standard_normal((5, L)) + 1j * rng.standard_normal((5, L))).astype(np.complex64)
    for inv in (False, True):
        got = T.fft_lines(a, inverse=inv)
        ref = np.fft.ifft(a.astype(np.complex128), axis=1) * L if inv else np.fft.fft(a.astype(np.complex128), axis=1)
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err < (1e-5 if L in BLUESTEIN else 2e-6), (L, inv, err)


def test_reference_phase(T):
    """parity_gabor.rs:40-70: per filter, response error < 1e-4 of its largest |r|; phase gradient error
    < 1e-3 rad/px on the pixels whose amplitude exceeds 5 % of the filter's largest."""
    g = golden("gabor")
    ref = T.reference_phase(g["img"])
    for k, (r, gx, gy, amp) in enumerate(ref):
        want = g["r_re"][k] + 1j * g["r_im"][k]
        max_amp = np.abs(want).max()
        assert np.abs(r - want).max() / max_amp < 1e-4
        strong = g["amp"][k] > 0.05 * max_amp
        assert strong.sum() > strong.size / 20
        assert np.abs(gx - g["gx"][k])[strong].max() < 1e-3
        assert np.abs(gy - g["gy"][k])[strong].max() < 1e-3
        assert np.abs(amp - g["amp"][k])[strong].max() < 1e-4 * max_amp
    # near the zeros of a response the gradient Im(conj r rx) / |r|^2 amplifies the float32 transforms' absolute
    # error e max|r| (e ~ 1e-6; the reference's Rust port has the same float32 transforms) by max|r|^2 / amp^2:
    # scaled by (amp / max)^2 the error stays below e times (the filter's frequency + 1) < 1e-5
    for k, (r, gx, gy, amp) in enumerate(ref):
        max_amp = np.abs(g["r_re"][k] + 1j * g["r_im"][k]).max()
        weak = g["amp"][k] > 1e-4 * max_amp
        err = np.maximum(np.abs(gx - g["gx"][k]), np.abs(gy - g["gy"][k]))
        assert (err * (g["amp"][k] / max_amp) ** 2)[weak].max() < 1e-5


def _gabor_bank_np(shape, cfg):
    """phaseflow.gabor_bank (python/optflow_ref/phaseflow.py:73-89), restated in numpy for the check."""
    h, w = shape
    fy = (np.fft.fftfreq(h) * 2 * np.pi)[:, None]
    fx = (np.fft.fftfreq(w) * 2 * np.pi)[None, :]
    s_hp = cfg.dc_cut * cfg.lam * max(cfg.scales) / (2 * np.pi)
    hp = 1.0 - np.exp(-(fx ** 2 + fy ** 2) * s_hp ** 2 / 2)
    bank = []
    for sc in cfg.scales:
        w0 = 2 * np.pi / (cfg.lam * sc)
        s = cfg.bandwidth * w0
        for k in range(cfg.n_orient):
            th = np.pi * k / cfg.n_orient
            bank.append(hp * np.exp(-((fx - w0 * np.cos(th)) ** 2 + (fy - w0 * np.sin(th)) ** 2) / (2 * s * s)))
    return bank


@pytest.mark.parametrize("shape", [(96, 128), (160, 224)])
def test_responses(T, oracle, shape):
    rng = np.random.default_rng(1)
    img = rng.random(shape).astype(np.float32)
    cfg = Config()
    got = T.responses(img, cfg)
    pad = np.pad(img.astype(np.float64), 32, mode="reflect")
    F2 = np.fft.fft2(pad)
    for k, G in enumerate(_gabor_bank_np(pad.shape, cfg)):
        r = np.fft.ifft2(F2 * G)
        want = oracle.bspline_coeffs(r.real) + 1j * oracle.bspline_coeffs(r.imag)
        err = np.abs(got[k] - want).max() / np.abs(want).max()
        assert err < 1e-4, (k, err)


@pytest.mark.parametrize("shape", [(2048, 2048), (2048, 136), (136, 2048)])
def test_responses_fixed_length(T, oracle, shape):
    """Padded length 2112 (2048-pixel sides, the benchmark's size) runs the transforms' compile-time plan and the
    staged column-pair / persistent row kernels; the mixed shapes pair it with a runtime plan on the other axis."""
    rng = np.random.default_rng(7)
    img = rng.random(shape).astype(np.float32)
    cfg = Config()
    got = T.responses(img, cfg)
    pad = np.pad(img.astype(np.float64), 32, mode="reflect")
    F2 = np.fft.fft2(pad)
    bank = _gabor_bank_np(pad.shape, cfg)
    for k in (0, 5, 11):
        r = np.fft.ifft2(F2 * bank[k])
        want = oracle.bspline_coeffs(r.real) + 1j * oracle.bspline_coeffs(r.imag)
        err = np.abs(got[k] - want).max() / np.abs(want).max()
        assert err < 1e-4, (shape, k, err)


@pytest.mark.parametrize("shape", [(2048, 2048), (136, 2048)])
def test_reference_phase_fixed_length(T, shape):
    """reference_phase (phaseflow.py:92-112) at padded length 2112 against a float64 numpy restatement: the
    response within 1e-4 of its largest |r|, the phase gradient within 1e-3 rad/px where the amplitude exceeds 5 %
    of the largest (the tolerances of parity_gabor.rs:40-70)."""
    rng = np.random.default_rng(8)
    img = rng.random(shape).astype(np.float32)
    cfg = Config()
    got = T.reference_phase(img, cfg)
    h, w = shape
    pad = np.pad(img.astype(np.float64), 32, mode="reflect")
    F2 = np.fft.fft2(pad)
    fy = (np.fft.fftfreq(pad.shape[0]) * 2 * np.pi)[:, None]
    fx = (np.fft.fftfreq(pad.shape[1]) * 2 * np.pi)[None, :]
    bank = _gabor_bank_np(pad.shape, cfg)
    crop = (slice(32, 32 + h), slice(32, 32 + w))
    for k in (0, 7):
        Z = F2 * bank[k]
        r = np.fft.ifft2(Z)[crop]
        rx = np.fft.ifft2(Z * 1j * fx)[crop]
        ry = np.fft.ifft2(Z * 1j * fy)[crop]
        a2 = np.abs(r) ** 2 + 1e-12
        gx, gy = (np.conj(r) * rx).imag / a2, (np.conj(r) * ry).imag / a2
        g_r, g_gx, g_gy, g_amp = got[k]
        max_amp = np.abs(r).max()
        assert np.abs(g_r - r).max() / max_amp < 1e-4
        strong = np.sqrt(a2) > 0.05 * max_amp
        assert strong.sum() > strong.size / 20
        assert np.abs(g_gx - gx)[strong].max() < 1e-3
        assert np.abs(g_gy - gy)[strong].max() < 1e-3
        assert np.abs(g_amp - np.sqrt(a2))[strong].max() < 1e-4 * max_amp


@pytest.mark.parametrize("order", [1, 2])
def test_local_solve(T, oracle, order):
    rng = np.random.default_rng(order)
    h, w = 70, 90
    gx, gy = rng.normal(size=(2, 12, h, w))
    wk = rng.uniform(0.1, 1.0, size=(12, h, w))
    c = rng.normal(size=(12, h, w)) + 20.0  # large right-hand sides, as with |u| ~ 25 px
    sums = [(wk * gx * gx).sum(0), (wk * gx * gy).sum(0), (wk * gy * gy).sum(0), (wk * gx * c).sum(0),
            (wk * gy * c).sum(0), (wk * c * c).sum(0), wk.sum(0)]
    sums[0][10:14, 10:14] = 0.0  # degenerate: no energy
    sums[1][10:14, 10:14] = 0.0
    sums[2][10:14, 10:14] = 0.0
    ux, uy = rng.normal(size=(2, h, w))
    got = T.local_solve(sums, ux, uy, Config(shape_order=order))
    want = oracle.local_solve(sums, ux, uy, 4.0, order)
    for a, b in zip(got, want):
        np.testing.assert_allclose(a, b, rtol=1e-7, atol=1e-9)


def test_median(T):
    rng = np.random.default_rng(5)
    for n in (1, 2, 3, 10, 1001, 4096, 100000):
        v = rng.exponential(size=n) * 1e3
        assert T.median(v) == np.median(v)
    v = np.repeat(rng.random(50), 7)
    assert T.median(v) == np.median(v)
    assert T.median(np.array([3.0, 1.0, 2.0, 2.0])) == 2.0
    # both signs; values clustered in one binade (a large bucket after two digits)
    for v in (rng.standard_normal(100001), 1.0 + rng.random(200000) * 1e-6):
        assert T.median(v) == np.median(v)
    # ties: a bucket within the candidate list, and beyond it (the remaining digits then take full passes), with
    # odd and even counts and the lower middle element inside or below the tied value
    for n_tie, n in ((30000, 100000), (150000, 200001), (150000, 200000), (60000, 120000)):
        v = rng.exponential(size=n)
        v[:n_tie] = np.median(v)
        rng.shuffle(v)
        assert T.median(v) == np.median(v), (n_tie, n)
    v = np.concatenate([np.zeros(60000), rng.random(60000)])
    assert T.median(v) == np.median(v)


def test_large_components(T, oracle):
    rng = np.random.default_rng(9)
    for p in (0.3, 0.5, 0.6):
        b = rng.random((123, 157)) < p
        for area in (5, 50, 327.68):
            np.testing.assert_array_equal(T.large_components(b, area), oracle.large_components(b, area))


@pytest.mark.parametrize("w2,h2,shift", [(260, 300, (0, 0)), (260, 300, (-7, 5)), (258, 301, (0, 0)),
                                         (64, 40, (3, -2)), (2048, 2048, (0, 0))])
def test_warp_tma_matches_gather(T, oracle, w2, h2, shift):
    """The TMA-staged warp (each 32 x 16 output tile's source box staged in shared memory) against the gather kernel
    bit for bit, and both against the oracle's B-spline sampler (interp.py:52-69): smooth fields up to 15 px, a band
    whose taps span more rows than the 64 x 40 box, positions beyond the plane (clamped, mirrored taps) and NaN
    positions. A plane whose row pitch is not a multiple of 16 bytes (258 floats) takes the gather kernel in both
    modes."""
    rng = np.random.default_rng(w2 + h2)
    c2 = rng.normal(size=(h2, w2)).astype(np.float32)
    h, w = h2 - 10, w2 + 6
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    sx = 15 * np.sin(xx / 37.0) * np.cos(yy / 53.0) + rng.normal(size=(h, w)) * 0.3
    sy = 9 * np.cos(xx / 29.0 + yy / 61.0)
    sy[h // 3:h // 3 + 5] += 60
    sx[5, 7] = np.nan
    sy[20, 30] = np.nan
    g, t0 = T.warp(c2, sx, sy, shift, mode=0)
    m, t1 = T.warp(c2, sx, sy, shift, mode=1)
    assert t0 == 0 and t1 == 0
    np.testing.assert_array_equal(m.view(np.uint32), g.view(np.uint32))
    X, Y = xx + shift[0] + sx, yy + shift[1] + sy
    ok = np.isfinite(X) & np.isfinite(Y)
    assert np.isnan(g[~ok]).all() and np.isfinite(g[ok]).all()
    ref = oracle.sample(c2.astype(np.float64), np.where(ok, X, 0), np.where(ok, Y, 0))
    np.testing.assert_allclose(g[ok], ref[ok], rtol=0, atol=1e-6)


@pytest.mark.parametrize("shape,amp", [((96, 128), 2.0), ((200, 264), 12.0), ((1024, 1024), 5.0)])
def test_accumulate_tma_matches_gather(T, shape, amp):
    """The TMA-staged accumulate (each filter pair's response box and reference-pack tile staged in shared memory)
    against the gather kernel, bit for bit, on refine's first inner iteration: a smooth start field, a sharp band whose
    blocks' taps span more than the 48 x 16-node box, a jump at the left border that moves taps outside the padded
    plane (mirrored indices)."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(shape[0])
    h, w = shape
    a = gaussian_filter(rng.random((h, w)), 1.5)
    b = np.roll(a, (1, 2), axis=(0, 1)) + 0.01 * rng.random((h, w))
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    ux = amp * np.sin(xx / 41.0) * np.cos(yy / 37.0)
    uy = amp * np.cos(xx / 29.0 + yy / 53.0)
    uy[h // 2:h // 2 + 3] += 40.0
    ux[:, :3] -= 80.0
    from optflow_b200.api import default_engine
    from optflow_b200.measure import Profile
    s0, t0 = T.accumulate(a, b, ux, uy, mode=0)
    prof = Profile(default_engine())
    prof.start()
    s1, t1 = T.accumulate(a, b, ux, uy, mode=1)
    assert "k_accumulate_tma" in prof.read()
    assert t0 == 0 and t1 == 0
    assert np.isfinite(s1).all()
    np.testing.assert_array_equal(s1, s0)


def test_atan2_phase(T):
    """The accumulate's float32 atan2 (common.cuh, a polynomial fit of atan on [0, 1]) within 5e-7 rad of the exact
    angle of its float32 arguments over 20 decades of magnitude and every direction, like CUDA's atan2f there; signed
    zeros and axes as atan2 gives them; NaN propagated."""
    rng = np.random.default_rng(17)
    n = 1 << 20
    mag = 10.0 ** rng.uniform(-20, 20, n)
    ang = rng.uniform(-np.pi, np.pi, n)
    x = (mag * np.cos(ang)).astype(np.float32)
    y = (mag * np.sin(ang)).astype(np.float32)
    special = np.array([(0.0, 0.0), (-0.0, 0.0), (0.0, -0.0), (-0.0, -0.0), (1, 0), (-1, 0), (0, 1), (0, -1), (1, 1),
                        (-1, 1), (1, -1), (-1, -1), (3, -0.0), (-3, -0.0), (1e-38, 1e-38), (1e-44, 2e-44),
                        (2e30, -1e30), (-5e-32, 7e-32)], np.float32)
    y = np.concatenate([y, special[:, 0]])
    x = np.concatenate([x, special[:, 1]])
    mine, cuda = T.atan2(y, x)
    exact = np.arctan2(y.astype(np.float64), x.astype(np.float64))
    assert np.abs(mine - exact).max() <= 5e-7
    assert np.abs(cuda - exact).max() <= 1e-6
    k = len(special)
    np.testing.assert_array_equal(np.signbit(mine[-k:]), np.signbit(exact[-k:]))
    m2, _ = T.atan2(np.array([np.nan, 1, np.nan], np.float32), np.array([1, np.nan, np.nan], np.float32))
    assert np.isnan(m2).all()


def test_prewarp_fill(T, oracle):
    """phaseflow.prewarp's fill (phaseflow.py:344-354) with scipy's nearest-source tie rule."""
    rng = np.random.default_rng(3)
    h, w = 90, 120
    low = np.zeros((h, w), bool)
    low[30:60, 40:80] = True
    low |= rng.random((h, w)) < 0.01
    ux, uy = rng.normal(size=(2, h, w))
    slope = rng.normal(size=(h, w, 4)) * 0.01
    R = Config().auto_edge_guard_px()
    gx, gy = T.prewarp_fill(low, ux, uy, slope, R)
    ok = oracle.edt(~low) > R
    _, (iy, ix) = oracle.edt(~ok, return_indices=True)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    dx, dy = xx - ix, yy - iy
    g = slope[iy, ix]
    ex = np.where(ok, ux, ux[iy, ix] + g[..., 0] * dx + g[..., 2] * dy)
    ey = np.where(ok, uy, uy[iy, ix] + g[..., 1] * dx + g[..., 3] * dy)
    np.testing.assert_allclose(gx, ex, rtol=0, atol=1e-12)
    np.testing.assert_allclose(gy, ey, rtol=0, atol=1e-12)


def test_render_matches_the_reference_generator(oracle):
    """ofc_synth_render against the reference's own renders (tests/golden/synth.npz) and, at 384 x 320 with a
    denser pattern, against the oracle's restatement: float64 images equal to 1e-12."""
    from optflow_b200 import synth
    from test_oracle import _synth_fields
    g = golden("synth")
    p = synth.make_pattern(64, 80, seed=3, rmin=1.5, rmax=2.5)
    for name, f in _synth_fields().items():
        assert np.abs(synth.render(p, 64, 80, f) - g[f"img_{name}"]).max() < 1e-12, name
    p = synth.make_pattern(320, 384, seed=5, rmin=1.5, rmax=4.0)
    for name, f in _synth_fields().items():
        assert np.abs(synth.render(p, 320, 384, f) - oracle.render(p, 320, 384, f)).max() < 1e-12, name


def test_render_with_grid_footing_and_bands(oracle):
    """The optional displacement terms of the renderer (a Gaussian-process grid, a footing settlement, finite shear
    bands) against the oracle's restatement, whose Newton inverse takes those terms' Jacobian by central differences:
    the two inverse maps meet at the same root, so the images agree to 1e-9."""
    from optflow_b200 import synth
    rng = np.random.default_rng(9)
    h, w = 288, 352
    grid, gx0, gy0 = synth.gp_grid(h, w, 96.0, 14.0, rng)
    f = synth.Field(grid=grid, gx0=gx0, gy0=gy0, footing=(3.0, 150.0, 140.0, 220.0, 40.0),
                    bands=[synth.Band((140.0, 40.0), (-0.7071067811865476, 0.7071067811865476), 6.0, 8.0, 180.0, 1.0),
                           synth.Band((220.0, 40.0), (0.7071067811865476, 0.7071067811865476), 6.0, 8.0, 180.0, 1.0)])
    p = synth.make_pattern(h, w, seed=4, rmin=1.5, rmax=2.5)
    assert np.abs(synth.render(p, h, w, f) - oracle.render(p, h, w, f)).max() < 1e-9


def test_fft_plan_orders_agree_and_tune():
    """Every factor order of a runtime plan computes the same transform (against numpy, as the default order), and
    the tuner returns an existing order per length."""
    from optflow_b200 import _abi, fftplan, testing
    lib = _abi.load()
    rng = np.random.default_rng(3)
    lengths = [320, 604, 1088]
    res = fftplan.tune(lengths, lines=256)
    for L in lengths:
        b, times = res[L]
        assert 0 <= b < lib.ofc_fft_plan_variants() and np.isfinite(times[b])
    x = (rng.normal(size=(8, 1088)) + 1j * rng.normal(size=(8, 1088))).astype(np.complex64)
    want = np.fft.fft(x.astype(np.complex128), axis=1)
    for v in range(lib.ofc_fft_plan_variants()):
        from optflow_b200 import Engine
        L = np.array([1088], np.int32)
        var = np.array([v], np.int32)
        lib.ofc_fft_set_plans(L.ctypes.data_as(_abi.c_i32_p), var.ctypes.data_as(_abi.c_i32_p), 1)
        got = testing.fft_lines(x, engine=Engine(0))  # a fresh engine builds its plan from the table
        assert np.abs(got - want).max() < 1e-5 * np.abs(want).max(), v
    zero = np.array([0], np.int32)
    lib.ofc_fft_set_plans(L.ctypes.data_as(_abi.c_i32_p), zero.ctypes.data_as(_abi.c_i32_p), 1)
    fftplan.install(force=True)  # the shipped table again
