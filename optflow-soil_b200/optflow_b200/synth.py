"""Synthetic speckle pairs with known displacement fields, rendered on the GPU (include/optflow_cuda_synth.h).

The blob draws follow the reference's generator call for call (python/optflow_ref/synth.py:20-29:
numpy default_rng(seed), uniform centres over the image plus a margin, uniform radii and amplitudes with
random sign), so a seed gives the reference's pattern; the rendering is the same analytic Gaussian-blob model
(synth.py:150-190: the same per-blob subsample rectangles, float64 throughout) evaluated by a CUDA kernel, so
render() returns the reference's float64 image to rounding; degrade() is synth.py:192-205 (noise, clip,
quantisation).
"""
import ctypes
from dataclasses import dataclass

import numpy as np

from ._abi import OfcField, c_double_p
from .api import _ptr, default_engine


@dataclass
class Pattern:
    cx: np.ndarray
    cy: np.ndarray
    r: np.ndarray
    a: np.ndarray


def make_pattern(h, w, seed=0, density=0.6, rmin=1.5, rmax=4.0, margin=80) -> Pattern:
    rng = np.random.default_rng(seed)
    rmean = 0.5 * (rmin + rmax)
    n = int(density * (h + 2 * margin) * (w + 2 * margin) / (np.pi * rmean ** 2))
    return Pattern(cx=rng.uniform(-margin, w + margin, n), cy=rng.uniform(-margin, h + margin, n),
                   r=rng.uniform(rmin, rmax, n), a=rng.uniform(0.3, 1.0, n) * rng.choice([-1.0, 1.0], n))


@dataclass
class Field:
    """x = c + A (X - c) + t + amp sin(2 pi X_x / wavelength) (sx, sy)."""
    A: tuple = ((1.0, 0.0), (0.0, 1.0))
    c: tuple = (0.0, 0.0)
    t: tuple = (0.0, 0.0)
    amp: float = 0.0
    wavelength: float = 256.0
    s: tuple = (1.0, 1.0)

    def ofc(self):
        f = OfcField()
        f.a00, f.a01 = self.A[0]
        f.a10, f.a11 = self.A[1]
        f.cx, f.cy = self.c
        f.tx, f.ty = self.t
        f.amp, f.wavelength = self.amp, self.wavelength
        f.sx, f.sy = self.s
        return f

    def displacement(self, h, w):
        """u(X) = x(X) - X on the reference grid."""
        yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
        dx, dy = xx - self.c[0], yy - self.c[1]
        s = self.amp * np.sin(2 * np.pi * xx / self.wavelength)
        x = self.c[0] + self.A[0][0] * dx + self.A[0][1] * dy + self.t[0] + s * self.s[0]
        y = self.c[1] + self.A[1][0] * dx + self.A[1][1] * dy + self.t[1] + s * self.s[1]
        return x - xx, y - yy


def uniform_strain(exx, eyy, center, exy=0.0, t=(0.0, 0.0)) -> Field:
    """synth.uniform_strain (python/optflow_ref/synth.py:84-85)."""
    return Field(A=((1 + exx, exy), (exy, 1 + eyy)), c=tuple(center), t=tuple(t))


def render(p: Pattern, h, w, field: Field = None, ss=4, engine=None) -> np.ndarray:
    eng = engine or default_engine()
    arrs = [np.ascontiguousarray(v, dtype=np.float64) for v in (p.cx, p.cy, p.r, p.a)]
    out = np.empty((h, w), np.float64)
    f = field.ofc() if field is not None else None
    eng._call("ofc_synth_render", *[_ptr(a, c_double_p) for a in arrs], len(p.cx), w, h, int(ss),
              ctypes.byref(f) if f is not None else None, _ptr(out, c_double_p))
    return out


def degrade(img, seed=0, noise=0.0, bits=None):
    """synth.degrade (python/optflow_ref/synth.py:192-205) without the illumination terms."""
    out = np.asarray(img, np.float64)
    if noise > 0:
        out = out + np.random.default_rng(seed).normal(0.0, noise, out.shape)
    out = np.clip(out, 0.0, 1.0)
    if bits:
        q = 2 ** bits - 1
        out = np.round(out * q) / q
    return out.astype(np.float32)


def polygon_mask(h, w, poly):
    """Pixels (x, y) inside a polygon [[x, y], ...] (even-odd rule at the pixel centres)."""
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    inside = np.zeros((h, w), bool)
    n = len(poly)
    for i in range(n):
        x1, y1 = poly[i]
        x2, y2 = poly[(i + 1) % n]
        crosses = (y1 > yy) != (y2 > yy)
        xint = (x2 - x1) * (yy - y1) / np.where(y2 != y1, y2 - y1, 1.0) + x1
        inside ^= crosses & (xx < xint)
    return inside


def rect_roi(h, w, x0, y0, x1, y1):
    """The ROI mask the reference CLI draws for the axis-aligned rectangle polygon [[x0, y0], [x1, y0], [x1, y1],
    [x0, y1]] (rust/crates/optflow-cli/src/polygon.rs:10-16, Pillow's scan-line filler, python/optflow_ref/io.py:155):
    vertices truncated toward zero, then every row from the top to the bottom vertex filled from the left to the
    right vertex, both ends inclusive."""
    m = np.zeros((h, w), bool)
    c0, r0, c1, r1 = int(x0), int(y0), int(x1), int(y1)
    m[max(r0, 0):min(r1 + 1, h), max(c0, 0):min(c1 + 1, w)] = True
    return m
