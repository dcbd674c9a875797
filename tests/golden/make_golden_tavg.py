"""Writes tests/golden/tavg.npz by running the reference's own Python temporal-averaging front-end
(python/optflow_ref/tavg.py) on seeded frames made with its generator (optflow_ref.synth).

Run in a checkout that has the reference: ``python tests/golden/make_golden_tavg.py [/path/to/reference]`` (or the
OPTFLOW_REFERENCE environment variable). Frames are rounded to float32 first (what the C ABI takes) and the reference runs on those values.
The reference's warp is scipy's cubic map_coordinates (mode "nearest"); the reference CLI and this engine warp with
the B-spline of interp::warp, so the two agree away from the image border, which is where the tests compare.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OPTFLOW_REFERENCE")
if not REF:
    sys.exit("usage: pass the reference checkout as the first argument (or set OPTFLOW_REFERENCE)")
sys.path.insert(0, os.path.join(REF, "python"))

from optflow_ref import synth, tavg  # noqa: E402
from optflow_ref.config import Config  # noqa: E402


def f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


def main():
    # five frames of a pattern drifting by (0.6, 0.3) px per frame, a little noise
    N = 128
    pat = synth.make_pattern(N, N, seed=3)
    rng = np.random.default_rng(4)
    fr = [f32(synth.render(pat, N, N, synth.Affine(np.eye(2), t=(0.6 * i, 0.3 * i), c=(N / 2, N / 2)))
              + 0.002 * rng.normal(size=(N, N))) for i in range(5)]
    cfg = Config(max_disp=8.0)
    aff0 = tavg.align_to(fr[2], fr[0], cfg)
    aff4 = tavg.align_to(fr[2], fr[4], cfg)
    # the right part moves (2 px), the left does not: the dense model follows it, the affine fit cannot
    f1 = f32(synth.render(pat, N, N, synth.Affine(np.eye(2), t=(2.0, 0.0), c=(N / 2, N / 2))))
    split = np.where(np.arange(N)[None, :] >= 70, f1, fr[0])
    dense = tavg.align_to(fr[0], split, Config(max_disp=8.0, tavg_model="dense"))
    # 192^2: the right half moves by 2 px, the left half does not; a mask keeps the affine fit to the right part
    M = 192
    pat2 = synth.make_pattern(M, M, seed=5)
    s0 = f32(synth.render(pat2, M, M))
    s1 = f32(synth.render(pat2, M, M, synth.Affine(np.eye(2), t=(2.0, 0.0), c=(M / 2, M / 2))))
    half = np.where(np.arange(M)[None, :] >= 96, s1, s0)
    mask = np.zeros((M, M), bool)
    mask[:, 112:] = True
    masked = tavg.align_to(s0, half, cfg, mask)
    unmasked = tavg.align_to(s0, half, cfg)
    plain = tavg.average_window(fr, 2)
    aligned = tavg.average_window(fr, 2, align=True, cfg=cfg)
    np.savez_compressed(os.path.join(HERE, "tavg.npz"), frames=np.float32(fr), split=np.float32(split),
                        m_static=np.float32(s0), m_half=np.float32(half), mask=mask.astype(np.uint8),
                        aff0=np.float32(aff0), aff4=np.float32(aff4), dense=np.float32(dense),
                        masked=np.float32(masked), unmasked=np.float32(unmasked), plain=np.float32(plain),
                        aligned=np.float32(aligned))
    print("tavg.npz written")


if __name__ == "__main__":
    main()
