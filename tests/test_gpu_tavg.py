"""The temporal-averaging front-end on the GPU (ofc_align_to, ofc_average_window) against the reference's
tavg.py (tests/golden/tavg.npz) and the CPU oracle's restatement of the reference CLI (tavg.rs).

Bars: aligned frames within 2e-3 of the reference away from the border (the engine's coarse grid agrees with the
reference's to ~1e-3 px, parity_poc.rs:50-51; the reference warps with scipy's map_coordinates, the CLI and the
engine with the B-spline of interp::warp, which agree away from the border); the plain mean bit for bit.
"""
import numpy as np
import pytest
from conftest import golden

from optflow_b200.config import Config
from optflow_b200.tavg import align_to, average_window

pytestmark = pytest.mark.gpu

M = (slice(20, -20), slice(20, -20))
TOL = 2e-3


@pytest.fixture(scope="module")
def g():
    return golden("tavg")


def test_align_to_affine_and_dense(g, oracle):
    cfg = Config(max_disp=8.0)
    fr = g["frames"]
    for c, o, want in ((fr[2], fr[0], g["aff0"]), (fr[2], fr[4], g["aff4"])):
        got = align_to(c, o, cfg)
        assert np.abs(got[M] - want[M]).max() < TOL
        assert np.abs(got[M] - oracle.align_to(c.astype(np.float64), o.astype(np.float64), cfg)[M]).max() < TOL
        assert np.abs(o[M] - c[M]).max() > 50 * TOL  # the frames did differ before the alignment
    dense = align_to(fr[0], g["split"], Config(max_disp=8.0, tavg_model="dense"))
    assert np.abs(dense[M] - g["dense"][M]).max() < TOL


def test_align_to_mask_restricts_the_fit(g):
    cfg = Config(max_disp=8.0)
    masked = align_to(g["m_static"], g["m_half"], cfg, mask=g["mask"].astype(bool))
    unmasked = align_to(g["m_static"], g["m_half"], cfg)
    assert np.abs(masked[M] - g["masked"][M]).max() < TOL
    assert np.abs(unmasked[M] - g["unmasked"][M]).max() < TOL
    right = (slice(20, -20), slice(120, -20))  # the moving part, inside the mask: the masked fit undoes its motion
    assert np.abs(masked[right] - g["m_static"][right]).max() < 5e-3
    assert np.abs(unmasked[right] - g["m_static"][right]).max() > 0.02


def test_align_to_returns_none_without_motion():
    flat = np.full((128, 128), 0.5, np.float32)
    assert align_to(flat, flat, Config(max_disp=8.0)) is None


def test_average_window(g, oracle):
    cfg = Config(max_disp=8.0)
    fr = g["frames"]
    np.testing.assert_array_equal(average_window(list(fr), 2), g["plain"])
    aligned = average_window(list(fr), 2, align=True, cfg=cfg)
    assert np.abs(aligned[M] - g["aligned"][M]).max() < TOL
    # the aligned mean keeps the centre frame's texture, the plain one blurs the drifting pattern (the frames
    # carry noise of 0.002, which bounds how close the aligned mean comes to the centre frame)
    e = lambda a: np.sqrt(np.mean((a[M] - fr[2][M]) ** 2))
    assert e(aligned) < 0.5 * e(g["plain"])
    # a frame whose motion cannot be estimated is left out, or with keep_unaligned enters as it is
    flat = np.full(fr[0].shape, 0.5, np.float32)
    f3 = [fr[2], flat]
    np.testing.assert_array_equal(average_window(f3, 0, align=True, cfg=cfg), fr[2])
    kept = average_window(f3, 0, align=True, cfg=cfg, keep_unaligned=True)
    np.testing.assert_array_equal(kept, np.float32((fr[2].astype(np.float64) + 0.5) / 2))
    with pytest.raises(ValueError, match="centre"):
        average_window(list(fr), 7)
    with pytest.raises(ValueError):
        align_to(fr[0], fr[1], Config(max_disp=8.0, tavg_model="linear"))
