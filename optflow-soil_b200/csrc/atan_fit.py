"""Coefficients of the float32 atan2 in common.cuh (atan2_phase): atan(a) = a P(a^2) on a in [0, 1], P of 8 terms
fitted to a minimax relative error of atan by iteratively reweighted least squares (Lawson's method) on Chebyshev-
distributed nodes in t = a^2.

    python optflow-soil_b200/csrc/atan_fit.py      # prints the coefficients and the errors of a float32 Horner
"""
import numpy as np


def fit(nterms=8, iters=80, nodes=4000):
    t = (1 - np.cos(np.linspace(0, np.pi, nodes))) / 2
    a = np.sqrt(t)
    f = np.where(a > 0, np.arctan(a) / np.where(a > 0, a, 1), 1.0)
    V = np.vander(t, nterms, increasing=True)
    w = np.ones_like(t)
    for _ in range(iters):
        c, *_ = np.linalg.lstsq(V * w[:, None], f * w, rcond=None)
        e = np.abs(V @ c - f) / f
        w = w * (e / e.max() + 1e-3) ** 0.5
        w /= w.max()
    return c


def float32_error(c, n=400001):
    a = np.linspace(0, 1, n)
    a32 = a.astype(np.float32)
    t32 = (a32 * a32).astype(np.float32)
    c32 = np.asarray(c, np.float32)
    h = np.full_like(t32, c32[-1])
    for k in range(len(c32) - 2, -1, -1):
        h = (h * t32 + c32[k]).astype(np.float32)
    p32 = (h * a32).astype(np.float32)
    return float(np.max(np.abs(p32.astype(np.float64) - np.arctan(a32.astype(np.float64)))))


if __name__ == "__main__":
    c = fit()
    print("coefficients (t^0 ... t^7):")
    for v in c:
        print(f"  {np.float32(v)!r:>16}   {v:.12e}")
    print("max |a P(a^2) - atan(a)|, float32 Horner:", float32_error(c))
