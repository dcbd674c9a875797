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
from dataclasses import field as dc_field

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
class Band:
    """A straight shear band (include/optflow_cuda_synth.h ofc_band): the material moves by
    0.5 delta (tanh(s / width) + bias) taper(a) along t, s = n . (X - e) across the band (n = (-t_y, t_x)),
    a = t . (X - e) along it; taper = 1 for length 0 (synth.ShearBand for bias 0), else a band of that length
    starting at e with tanh ends."""
    e: tuple
    t: tuple
    delta: float
    width: float
    length: float = 0.0
    bias: float = 0.0


@dataclass
class Field:
    """x = c + A (X - c) + t + amp sin(2 pi X_x / wavelength) (sx, sy) + the optional terms of ofc_field:
    grid (2, gny, gnx) cubic B-spline coefficients at (gx0 + i gh, gy0 + j gh); footing = (fs, fdecay, fx0, fx1, fy):
    u_y += fs exp(-d / fdecay), d the distance to the segment (fx0, fy)-(fx1, fy); bands: up to 4 Band."""
    A: tuple = ((1.0, 0.0), (0.0, 1.0))
    c: tuple = (0.0, 0.0)
    t: tuple = (0.0, 0.0)
    amp: float = 0.0
    wavelength: float = 256.0
    s: tuple = (1.0, 1.0)
    grid: np.ndarray = None
    gx0: float = 0.0
    gy0: float = 0.0
    gh: float = 16.0
    footing: tuple = None
    bands: list = dc_field(default_factory=list)

    def ofc(self):
        f = OfcField()
        f.a00, f.a01 = self.A[0]
        f.a10, f.a11 = self.A[1]
        f.cx, f.cy = self.c
        f.tx, f.ty = self.t
        f.amp, f.wavelength = self.amp, self.wavelength
        f.sx, f.sy = self.s
        if self.grid is not None:
            g = np.ascontiguousarray(self.grid, dtype=np.float64)
            f._keep = g  # the struct points into this array
            f.grid = g.ctypes.data_as(c_double_p)
            f.gny, f.gnx = g.shape[1], g.shape[2]
            f.gx0, f.gy0, f.gh = self.gx0, self.gy0, self.gh
        if self.footing is not None:
            f.fs, f.fdecay, f.fx0, f.fx1, f.fy = self.footing
        if len(self.bands) > 4:
            raise ValueError("at most 4 shear bands")
        f.n_bands = len(self.bands)
        for k, b in enumerate(self.bands):
            f.bands[k].ex, f.bands[k].ey = b.e
            f.bands[k].tx, f.bands[k].ty = b.t
            f.bands[k].delta, f.bands[k].width, f.bands[k].length, f.bands[k].bias = b.delta, b.width, b.length, b.bias
        return f

    def extra(self, X, Y):
        """The optional terms' displacement (ux, uy) at reference points X, Y (float64 arrays)."""
        ux, uy = np.zeros_like(X), np.zeros_like(X)
        if self.grid is not None:
            g = np.asarray(self.grid, np.float64)
            gny, gnx = g.shape[1:]
            gx, gy = (X - self.gx0) / self.gh, (Y - self.gy0) / self.gh
            fx, fy = np.floor(gx), np.floor(gy)
            wx, wy = _bspline_w(gx - fx), _bspline_w(gy - fy)
            ix, iy = fx.astype(np.int64), fy.astype(np.int64)
            for a in range(4):
                r = np.clip(iy - 1 + a, 0, gny - 1)
                for b in range(4):
                    c = np.clip(ix - 1 + b, 0, gnx - 1)
                    w = wy[a] * wx[b]
                    ux += w * g[0][r, c]
                    uy += w * g[1][r, c]
        if self.footing is not None:
            fs, fdecay, fx0, fx1, fy = self.footing
            d = np.hypot(X - np.clip(X, fx0, fx1), Y - fy)
            uy += fs * np.exp(-d / fdecay)
        for b in self.bands:
            rx, ry = X - b.e[0], Y - b.e[1]
            sv = -b.t[1] * rx + b.t[0] * ry
            av = b.t[0] * rx + b.t[1] * ry
            tp = 1.0 if b.length <= 0 else 0.25 * (1 + np.tanh(av / b.width)) * (1 + np.tanh((b.length - av) / b.width))
            v = 0.5 * b.delta * (np.tanh(sv / b.width) + b.bias) * tp
            ux += v * b.t[0]
            uy += v * b.t[1]
        return ux, uy

    def displacement_at(self, X, Y):
        """u(X) = x(X) - X at reference points X, Y (float64 arrays)."""
        X, Y = np.asarray(X, np.float64), np.asarray(Y, np.float64)
        dx, dy = X - self.c[0], Y - self.c[1]
        s = self.amp * np.sin(2 * np.pi * X / self.wavelength)
        x = self.c[0] + self.A[0][0] * dx + self.A[0][1] * dy + self.t[0] + s * self.s[0]
        y = self.c[1] + self.A[1][0] * dx + self.A[1][1] * dy + self.t[1] + s * self.s[1]
        ex, ey = self.extra(X, Y)
        return x + ex - X, y + ey - Y

    def displacement(self, h, w):
        """u(X) = x(X) - X on the reference grid."""
        yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
        return self.displacement_at(xx, yy)


def _bspline_w(t):
    s = 1.0 - t
    t2 = t * t
    return (s * s * s / 6.0, (3.0 * t2 * t - 6.0 * t2 + 4.0) / 6.0, (-3.0 * t2 * t + 3.0 * t2 + 3.0 * t + 1.0) / 6.0,
            t2 * t / 6.0)


def gp_grid(h, w, length, amp, rng, gh=16.0, margin=64.0):
    """A smooth random displacement field as B-spline coefficients (2, gny, gnx) at spacing gh over the image plus a
    margin: white noise filtered by a Gaussian of standard deviation `length` (a Gaussian-process sample with a
    squared-exponential covariance of that length scale), scaled so that its largest |u| on the grid is `amp`.
    Returns (grid, gx0, gy0) for Field(grid=..., gx0=..., gy0=..., gh=gh)."""
    gnx = int(np.ceil((w + 2 * margin) / gh)) + 1
    gny = int(np.ceil((h + 2 * margin) / gh)) + 1
    sig = length / gh
    py, px = max(gny, int(4 * sig) + gny), max(gnx, int(4 * sig) + gnx)
    ky = np.fft.fftfreq(py)[:, None]
    kx = np.fft.fftfreq(px)[None, :]
    gauss = np.exp(-2.0 * (np.pi * sig) ** 2 * (kx * kx + ky * ky))
    out = np.empty((2, gny, gnx))
    for c in range(2):
        noise = rng.normal(0.0, 1.0, (py, px))
        out[c] = np.real(np.fft.ifft2(np.fft.fft2(noise) * gauss))[:gny, :gnx]
    mag = np.sqrt(out[0] ** 2 + out[1] ** 2).max()
    out *= amp / max(mag, 1e-30)
    return out, -margin, -margin


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


def footing_field(k, w=1920, h=1080, surface=300.0, width=240.0, rate=0.05, decay=150.0, slip=12.0, frames=600,
                  band_width=8.0, band_length=360.0):
    """Frame k of a rigid strip footing settling into sand: the footing (width px, centred, its base on the sand
    surface y = surface) settles by rate * k px; the sand below moves down by that settlement times exp(-d / decay),
    d the distance to the footing base; two symmetric shear bands leave the footing edges at 45 degrees downward and
    outward (tanh profile of width band_width, band_length px long) and carry a tangential slip growing linearly to
    `slip` px at the last frame."""
    x0, x1 = w / 2 - width / 2, w / 2 + width / 2
    s = rate * k
    d = slip * k / max(frames - 1, 1)
    r = 0.7071067811865476
    bands = [Band(e=(x0, surface), t=(-r, r), delta=d, width=band_width, length=band_length),
             Band(e=(x1, surface), t=(r, r), delta=d, width=band_width, length=band_length)]
    return Field(footing=(s, decay, x0, x1, surface), bands=bands)
