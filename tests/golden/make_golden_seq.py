"""Writes tests/golden/seq.npz by running the reference's own Python track_sequence (chain mode,
python/optflow_ref/track.py:260-315) on seeded frames made with its generator (optflow_ref.synth).

Run in a checkout that has the reference: ``python tests/golden/make_golden_seq.py [/path/to/reference]`` (or the
OPTFLOW_REFERENCE environment variable). Frames are rounded to float32 first (what the C ABI takes) and the reference runs on those values.
Two runs: the default ref_update_conf (the reference stays at frame 0) and ref_update_conf = 0.995 (the reference
moves to k - 1 at every frame from k = 2 on), both with an ROI.
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


def f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


def main():
    n, K = 128, 4
    pat = synth.make_pattern(n, n, seed=21)
    fr = [f32(synth.degrade(synth.render(pat, n, n, synth.uniform_strain(0.004 * j, -0.002 * j, (n / 2, n / 2),
                                                                          t=(0.7 * j, 0.4 * j))),
                            seed=j, noise=0.005, bits=8)) for j in range(K)]
    roi = np.zeros((n, n), bool)
    roi[12:-12, 16:-16] = True
    out = dict(frames=np.float32(fr), roi=roi.astype(np.uint8))
    for tag, ruc in (("a", 0.5), ("b", 0.995)):
        t = time.time()
        for k, r in track.track_sequence(fr, Config(ref_update_conf=ruc), mask=roi):
            for q in ("ux", "uy", "conf", "raw_ux", "raw_uy"):
                out[f"{tag}{k}_{q}"] = np.float32(getattr(r, q))
            for q in ("Exx", "Eyy", "Exy", "gmax", "vol"):
                out[f"{tag}{k}_{q}"] = np.float32(r.strain[q])
            out[f"{tag}{k}_ref"] = np.int32(r.timing["reference"])
            out[f"{tag}{k}_mean"] = np.float64(r.timing["mean_conf"])
        print(f"run {tag}: {time.time() - t:.1f} s")
    np.savez_compressed(os.path.join(HERE, "seq.npz"), **out)
    print("seq.npz written")


if __name__ == "__main__":
    main()
