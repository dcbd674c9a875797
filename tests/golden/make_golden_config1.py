"""Writes tests/golden/config1.npz: the reference's own chain-mode track_sequence (python/optflow_ref/track.py:
260-315) on the CPU-runnable sequence the benchmark configuration names first: five uint8 256 x 256 frames of
synth.make_pattern(256, 256, seed=1), frame k under a uniform strain exx = 0.005 k about (128, 128) plus the
translation (0.8 k, 0) px, rendered and degraded with Gaussian noise 0.005 (seed k) to 8 bits; default
configuration, no ROI.

Stored per frame: ux, uy, conf, Exx, Eyy, Exy, gmax and vol in full (float32); the reference index and mean
confidence.

Run in a checkout that has the reference: ``python tests/golden/make_golden_config1.py [/path/to/reference]``
(or the OPTFLOW_REFERENCE environment variable).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OPTFLOW_REFERENCE")
if not REF:
    sys.exit("usage: pass the reference checkout as the first argument (or set OPTFLOW_REFERENCE)")
sys.path.insert(0, os.path.join(REF, "python"))

from optflow_ref import synth, track  # noqa: E402
from optflow_ref.config import Config  # noqa: E402


def main():
    n = 256
    pat = synth.make_pattern(n, n, seed=1)
    frames = []
    for k in range(5):
        img = synth.render(pat, n, n, synth.uniform_strain(0.005 * k, 0.0, (128, 128), t=(0.8 * k, 0.0)))
        frames.append(np.round(synth.degrade(img, seed=k, noise=0.005, bits=8) * 255).astype(np.uint8))
    grey = [f.astype(np.float64) / 255.0 for f in frames]
    out = {"frames": np.stack(frames)}
    t = time.time()
    for k, r in track.track_sequence(grey, Config()):
        out[f"f{k}_ux"], out[f"f{k}_uy"], out[f"f{k}_conf"] = (np.float32(getattr(r, q)) for q in ("ux", "uy", "conf"))
        for q in ("Exx", "Eyy", "Exy", "gmax", "vol"):
            out[f"f{k}_{q}"] = np.float32(r.strain[q])
        out[f"f{k}_meta"] = np.array([r.timing["reference"], r.timing["mean_conf"]])
        print(k, f"{time.time() - t:.1f} s", flush=True)
    np.savez_compressed(os.path.join(HERE, "config1.npz"), **out)
    print("config1.npz written")


if __name__ == "__main__":
    main()
