"""Writes tests/golden/iter.npz from the reference's own frame iterator with temporal averaging
(python/optflow_ref/io.py:100-153, iter_frames / _iter_averaged, over tavg.average_window): ten 288 x 256 uint8 frames
of a drifting pattern made with its generator (optflow_ref.synth), handed to the reference in memory (its frame
reader replaced by a list lookup, each frame through its own to_gray as read_image would), downscaled by 2.

Cases: (plain) tavg 0, start 2, stop 9, step 3; (edge) tavg 2, start 1, step 3, to the end of the input, so the last
windows are one-sided and aligned with the dense model; (aligned) tavg 1, start 0, stop 7, step 2, every window
aligned with the affine model inside a mask.

Run in a checkout that has the reference: ``python tests/golden/make_golden_iter.py [/path/to/reference]``
(or the OPTFLOW_REFERENCE environment variable).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OPTFLOW_REFERENCE")
if not REF:
    sys.exit("usage: pass the reference checkout as the first argument (or set OPTFLOW_REFERENCE)")
sys.path.insert(0, os.path.join(REF, "python"))

from optflow_ref import io, synth  # noqa: E402
from optflow_ref.config import Config  # noqa: E402


def main():
    h, w = 288, 256
    pat = synth.make_pattern(h, w, seed=41)
    frames = []
    for i in range(10):
        img = synth.render(pat, h, w, synth.Affine(np.eye(2), t=(0.8 * i, 0.5 * i), c=(w / 2, h / 2)))
        frames.append(np.round(synth.degrade(img, seed=i, noise=0.004, bits=8) * 255).astype(np.uint8))
    grey = [io.to_gray(f) for f in frames]
    io._raw_frames = lambda source, lo, hi: iter(grey[lo:hi])
    io.list_images = lambda source: list(range(len(grey)))
    io.read_image = lambda p: grey[p]
    mask = np.zeros((h // 2, w // 2), bool)
    mask[10:-10, 20:-20] = True
    cfg = Config(max_disp=8.0)
    out = {"frames": np.stack(frames), "mask": mask.astype(np.uint8)}
    cases = {
        "plain": dict(start=2, stop=9, step=3, scale=2),
        "edge": dict(start=1, step=3, scale=2, tavg=2, cfg=cfg),
        "aligned": dict(start=0, stop=7, step=2, scale=2, tavg=1, align=True, cfg=cfg, mask_fn=lambda shape: mask),
    }
    for name, kw in cases.items():
        got = list(io.iter_frames("frames", **kw))
        out[name] = np.stack(got).astype(np.float32)
        print(name, len(got))
    np.savez_compressed(os.path.join(HERE, "iter.npz"), **out)
    print("iter.npz written")


if __name__ == "__main__":
    main()
