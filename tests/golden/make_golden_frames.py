"""Writes tests/golden/frames.npz from the reference's own frame front-end (python/optflow_ref/io.py:15-51,
to_gray and downscale): seeded 37 x 29 images of every pixel format the engine takes (uint8 grey, RGB, RGBA; uint16
grey and RGB; float32 grey), their grey levels (float64) and their box downscales by 2 and 3.

Run in a checkout that has the reference: ``python tests/golden/make_golden_frames.py [/path/to/reference]``
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

from optflow_ref import io  # noqa: E402


def main():
    rng = np.random.default_rng(31)
    h, w = 37, 29
    imgs = {
        "gray8": rng.integers(0, 256, (h, w), dtype=np.uint8),
        "rgb24": rng.integers(0, 256, (h, w, 3), dtype=np.uint8),
        "rgba32": rng.integers(0, 256, (h, w, 4), dtype=np.uint8),
        "gray16": rng.integers(0, 65536, (h, w), dtype=np.uint16),
        "rgb48": rng.integers(0, 65536, (h, w, 3), dtype=np.uint16),
        "f32": rng.random((h, w), dtype=np.float32),
    }
    out = {}
    for name, a in imgs.items():
        g = io.to_gray(a if name != "rgba32" else a[..., :3])  # the reference's colour path takes R, G, B
        out[f"{name}_in"] = a
        out[f"{name}_gray"] = g
        for s in (2, 3):
            out[f"{name}_down{s}"] = io.downscale(g, s)
    np.savez_compressed(os.path.join(HERE, "frames.npz"), **out)
    print("frames.npz written")


if __name__ == "__main__":
    main()
