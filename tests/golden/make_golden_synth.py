"""Writes tests/golden/synth.npz with the reference's own generator (python/optflow_ref/synth.py): a pattern from
make_pattern, its render with no field, under uniform_strain, and under an affine map plus a sinusoid along x (the
field of the 2048^2 benchmark pair, which synth.py has no class for: it is built here on synth.Affine, with the
inverse map by Newton steps from the affine inverse), and degrade() of each (noise 0.01, 8 bits).

Run in a checkout that has the reference: ``python tests/golden/make_golden_synth.py <reference checkout>`` (or the
OPTFLOW_REFERENCE environment variable).
"""
import os
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OPTFLOW_REFERENCE")
if not REF:
    sys.exit("usage: pass the reference checkout as the first argument (or set OPTFLOW_REFERENCE)")
sys.path.insert(0, os.path.join(REF, "python"))
from optflow_ref import synth  # noqa: E402


class SinAffine(synth.Affine):
    """x = c + A (X - c) + t + amp sin(2 pi X / wavelength) (sx, sy)."""

    def __init__(self, A, t, c, amp, wavelength, s):
        super().__init__(A, t, c)
        self.amp, self.wavelength, self.s = amp, wavelength, np.asarray(s, dtype=np.float64)

    def fwd(self, X, Y):
        x, y = super().fwd(X, Y)
        s = self.amp * np.sin(2 * np.pi * X / self.wavelength)
        return x + s * self.s[0], y + s * self.s[1]

    def inv(self, x, y):
        X, Y = super().inv(x, y)
        A = self.A
        for _ in range(30):
            fx, fy = self.fwd(X, Y)
            fx, fy = fx - x, fy - y
            ds = self.amp * (2 * np.pi / self.wavelength) * np.cos(2 * np.pi * X / self.wavelength)
            j00, j01, j10, j11 = A[0, 0] + ds * self.s[0], A[0, 1], A[1, 0] + ds * self.s[1], A[1, 1]
            d = j00 * j11 - j01 * j10
            sx, sy = (j11 * fx - j01 * fy) / d, (-j10 * fx + j00 * fy) / d
            X, Y = X - sx, Y - sy
            if np.max(np.abs(sx) + np.abs(sy)) < 1e-13:
                break
        return X, Y


def main():
    h, w = 64, 80
    p = synth.make_pattern(h, w, seed=3, rmin=1.5, rmax=2.5)
    fields = {
        "none": None,
        "strain": synth.uniform_strain(0.01, -0.004, (40.0, 32.0), exy=0.003, t=(1.3, -0.7)),
        "sinaff": SinAffine([[1.01, 0.003], [0.003, 0.996]], (0.4, -0.25), (40.0, 32.0), 1.5, 32.0, (1.0, 1.0)),
    }
    out = {"cx": p.cx, "cy": p.cy, "r": p.r, "a": p.a}
    for i, (name, f) in enumerate(fields.items()):
        img = synth.render(p, h, w, f)
        out[f"img_{name}"] = img
        out[f"deg_{name}"] = synth.degrade(img, seed=10 + i, noise=0.01, bits=8)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "synth.npz")
    np.savez_compressed(path, **out)
    print(path, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
