"""Writes tests/golden/config2.npz and tests/golden/poc_peaks.npz with the reference's own Python
(python/optflow_ref): the 2048^2 benchmark pair and the integer POC peaks of its coarse stage.

config2.npz -- the 2048 x 2048 pair of the benchmark, made by the reference's generator: make_pattern(2048, 2048,
seed=7, rmin=1.5, rmax=2.5) (mean speckle diameter about 4 px), image 1 the undeformed render, image 2 the render
under x = c + A (X - c) + 1.5 sin(2 pi X / 256) (1, 1), A = [[1.01, 0.003], [0.003, 0.996]], c = (1024, 1024)
(exx 0.01, eyy -0.004, gxy 0.006), both degraded with noise 0.01 (seeds 1 and 2) and 8 bits; the ROI is the
reference's io.polygon_mask of the square [204.8, 1843.2]^2 (the central 80 %). The frames themselves are not
stored (8 MiB): their SHA-256 and per-row sums are, so a test can prove that a renderer gave the same uint8 frames.
Also stored: the reference's coarse_flow (poc.py:216-239) grid after clean (ux, uy, peak) and the integer peak of
every grid point of both pyramid levels.

poc_peaks.npz -- the integer peaks of the reference's coarse_flow on its own POC fixtures (poc_a/poc_b with the
default configuration, the strip pair with max_disp 100: two levels).

The integer peak of a grid point is the window offset round(d) plus the argmax of the last shifted correlation
surface evaluated there minus the half window (poc.py:50, 82-88). It is read from the reference's own poc_shift
by wrapping np.unravel_index while poc_grid runs; the grid point and offset come from poc_grid's frame.

Run in a checkout that has the reference: ``python tests/golden/make_golden_config2.py <reference checkout>`` (or the
OPTFLOW_REFERENCE environment variable). Takes a few minutes (the Python renderer at 2048^2).
"""
import hashlib
import os
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OPTFLOW_REFERENCE")
if not REF:
    sys.exit("usage: pass the reference checkout as the first argument (or set OPTFLOW_REFERENCE)")
sys.path.insert(0, os.path.join(REF, "python"))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from optflow_ref import poc, synth  # noqa: E402
from optflow_ref.config import Config  # noqa: E402
from optflow_ref.io import polygon_mask  # noqa: E402

from make_golden_synth import SinAffine  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(REF, "rust", "crates", "optflow-core", "tests", "fixtures")


def coarse_with_peaks(a, b, cfg):
    """The reference's coarse_flow, and per pyramid level (level 0 first) the (ny, nx, 2) integer peaks."""
    levels = []
    orig_grid, orig_shift, orig_unravel = poc.poc_grid, poc.poc_shift, np.unravel_index
    last = {}

    def unravel(idx, shape):
        r = orig_unravel(idx, shape)
        last["am"] = (int(r[0]), int(r[1]))
        return r

    def shift(wa, wb):
        out = orig_shift(wa, wb)
        f = sys._getframe(1).f_locals
        iy, ix = last["am"]
        h, w = wa.shape
        levels[-1][f["i"], f["j"]] = (f["ox"] + ix - w // 2, f["oy"] + iy - h // 2)
        return out

    def grid(I1, I2, xs, ys, win, init=None, iters=3):
        levels.append(np.full((len(ys), len(xs), 2), np.iinfo(np.int32).min, np.int64))
        return orig_grid(I1, I2, xs, ys, win, init, iters)

    poc.poc_grid, poc.poc_shift, np.unravel_index = grid, shift, unravel
    try:
        g = poc.coarse_flow(a, b, cfg)
    finally:
        poc.poc_grid, poc.poc_shift, np.unravel_index = orig_grid, orig_shift, orig_unravel
    return g, [lv.astype(np.int32) for lv in reversed(levels)]


def fixtures():
    out = {}
    a, b = np.load(os.path.join(FIX, "poc_a.npy")).astype(np.float64), np.load(os.path.join(FIX, "poc_b.npy"))
    _, lv = coarse_with_peaks(a, b.astype(np.float64), Config())
    for k, p in enumerate(lv):
        out[f"grid_l{k}"] = p
    sa, sb = np.load(os.path.join(FIX, "poc_strip_a.npy")), np.load(os.path.join(FIX, "poc_strip_b.npy"))
    _, lv = coarse_with_peaks(sa.astype(np.float64), sb.astype(np.float64), Config(max_disp=100))
    for k, p in enumerate(lv):
        out[f"strip_l{k}"] = p
    path = os.path.join(HERE, "poc_peaks.npz")
    np.savez_compressed(path, **out)
    print(path, {k: v.shape for k, v in out.items()})


def config2():
    n = 2048
    p = synth.make_pattern(n, n, seed=7, rmin=1.5, rmax=2.5)
    c = n / 2.0
    field = SinAffine([[1.01, 0.003], [0.003, 0.996]], (0.0, 0.0), (c, c), 1.5, 256.0, (1.0, 1.0))
    a = synth.degrade(synth.render(p, n, n, None), seed=1, noise=0.01, bits=8)
    b = synth.degrade(synth.render(p, n, n, field), seed=2, noise=0.01, bits=8)
    qa, qb = np.round(a * 255).astype(np.uint8), np.round(b * 255).astype(np.uint8)
    lo, hi = 0.1 * n, 0.9 * n
    roi = polygon_mask((n, n), [[lo, lo], [hi, lo], [hi, hi], [lo, hi]])
    # the engine and the CLI read 8-bit frames as float32 levels / 255; POC runs on those values in float64
    g, lv = coarse_with_peaks((qa / 255.0).astype(np.float32).astype(np.float64),
                              (qb / 255.0).astype(np.float32).astype(np.float64), Config())
    out = {"sha_a": np.array(hashlib.sha256(qa.tobytes()).hexdigest()),
           "sha_b": np.array(hashlib.sha256(qb.tobytes()).hexdigest()),
           "rows_a": qa.sum(axis=1, dtype=np.int64), "rows_b": qb.sum(axis=1, dtype=np.int64),
           "roi": np.packbits(roi), "xs": g.xs, "ys": g.ys, "ux": g.ux, "uy": g.uy, "peak": g.peak}
    for k, pk in enumerate(lv):
        out[f"ipk_l{k}"] = pk
    path = os.path.join(HERE, "config2.npz")
    np.savez_compressed(path, **out)
    print(path, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    fixtures()
    config2()
