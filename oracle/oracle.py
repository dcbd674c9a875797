"""numpy front end of the CPU oracle (oracle.cpp), for the tests and the benchmark's CPU baseline.

TEST INFRASTRUCTURE: the checker of the CUDA engine, never part of it. Function names and
conventions follow the reference's Python specification (python/optflow_ref/*.py): images are
float64 arrays indexed [row, col], displacement fields (ux, uy) in pixels.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboptflow_oracle.so")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _cfg(cfg):
    from optflow_b200.config import Config
    c = (cfg or Config()).to_ofc()
    return ctypes.byref(c), c


def threads(n=0):
    return lib().oro_threads(int(n))


def fft2(a, inverse=False):
    z = np.ascontiguousarray(a, dtype=np.complex128).copy()
    h, w = z.shape
    lib().oro_fft2(_p(z), w, h, int(inverse))
    return z


def bspline_coeffs(img):
    a = _d(img)
    out = np.empty_like(a)
    lib().oro_bspline_coeffs(_p(a), _p(out), a.shape[1], a.shape[0])
    return out


def sample(coeffs, x, y):
    c = _d(coeffs)
    x, y = np.broadcast_arrays(_d(x), _d(y))
    x, y = _d(x), _d(y)
    out = np.empty(x.shape)
    lib().oro_sample(_p(c), c.shape[1], c.shape[0], _p(x), _p(y), ctypes.c_size_t(x.size), _p(out))
    return out


def gauss_blur(a, sigma):
    a = _d(a)
    out = np.empty_like(a)
    lib().oro_gauss_blur(_p(a), _p(out), a.shape[1], a.shape[0], ctypes.c_double(sigma))
    return out


def edt(inp, return_indices=False):
    """scipy.ndimage.distance_transform_edt(inp[, return_indices=True])."""
    b = np.ascontiguousarray(inp != 0, dtype=np.uint8)
    h, w = b.shape
    dist = np.empty((h, w))
    idx = np.empty((h, w), np.int64) if return_indices else None
    lib().oro_edt(_p(b), w, h, _p(dist), _p(idx))
    if not return_indices:
        return dist
    return dist, (idx // w, idx % w)


def large_components(b, min_area):
    a = np.ascontiguousarray(b, dtype=np.uint8)
    out = np.empty_like(a)
    lib().oro_large_components(_p(a), a.shape[1], a.shape[0], ctypes.c_double(min_area), _p(out))
    return out.astype(bool)


def reference_phase(I1, cfg=None):
    """phaseflow.reference_phase: list of (r, gx, gy, amp) per filter."""
    a = _d(I1)
    h, w = a.shape
    pc, c = _cfg(cfg)
    F = c.n_orient * c.n_scales
    planes = [np.empty((F, h, w)) for _ in range(5)]
    lib().oro_reference_phase(_p(a), w, h, pc, *[_p(p) for p in planes])
    re, im, gx, gy, amp = planes
    return [(re[k] + 1j * im[k], gx[k], gy[k], amp[k]) for k in range(F)]


def local_solve(sums, ux, uy, sigma, order):
    """phaseflow.local_solve on the seven per-pixel sums: (ux, uy, energy, resid, slope)."""
    s = _d(np.stack(sums))
    ux, uy = _d(ux), _d(uy)
    h, w = ux.shape
    out = [np.empty((h, w)) for _ in range(4)]
    slope = np.empty((h, w, 4))
    lib().oro_local_solve(_p(s), _p(ux), _p(uy), w, h, ctypes.c_double(sigma), int(order),
                          *[_p(o) for o in out], _p(slope))
    return (*out, slope)


def refine(I1, I2, ux, uy, cfg=None):
    """phaseflow.refine: dict(ux, uy, conf, resid, energy)."""
    a, b, ux, uy = _d(I1), _d(I2), _d(ux), _d(uy)
    h, w = a.shape
    pc, _ = _cfg(cfg)
    out = [np.empty((h, w)) for _ in range(5)]
    lib().oro_refine(_p(a), _p(b), w, h, _p(ux), _p(uy), pc, *[_p(o) for o in out])
    return dict(zip(("ux", "uy", "conf", "resid", "energy"), out))


def first_sums(I1, I2, ux, uy, cfg=None):
    """The seven per-pixel sums of refine's first inner iteration (pre-warp = blur of the start field)."""
    a, b, ux, uy = _d(I1), _d(I2), _d(ux), _d(uy)
    h, w = a.shape
    pc, _ = _cfg(cfg)
    out = np.empty((7, h, w))
    lib().oro_first_sums(_p(a), _p(b), w, h, _p(ux), _p(uy), pc, _p(out))
    return out


def set_f32_storage(on):
    """Round responses and reference pack to float32 (the Rust port's storage) in the oracle's refine."""
    lib().oro_set_f32_storage(int(bool(on)))


def poc_shift(a, b):
    a, b = _d(a), _d(b)
    out = np.empty(3)
    lib().oro_poc_shift(_p(a), _p(b), a.shape[1], a.shape[0], _p(out))
    return float(out[0]), float(out[1]), float(out[2])


def n_levels(max_disp, win, shape):
    return lib().oro_n_levels(ctypes.c_double(max_disp), int(win), int(shape[0]), int(shape[1]))


def level_window(shape, win):
    wy, wx = ctypes.c_int(), ctypes.c_int()
    ok = lib().oro_level_window(int(shape[0]), int(shape[1]), int(win), ctypes.byref(wy), ctypes.byref(wx))
    return (wy.value, wx.value) if ok else None


def poc_grid(I1, I2, xs, ys, win, init=None):
    """poc.poc_grid (no clean): (ux, uy, peak) of shape (ny, nx)."""
    a, b = _d(I1), _d(I2)
    h, w = a.shape
    wy, wx = (win, win) if np.isscalar(win) else win
    xs = np.ascontiguousarray(xs, dtype=np.int32)
    ys = np.ascontiguousarray(ys, dtype=np.int32)
    ny, nx = len(ys), len(xs)
    out = [np.empty((ny, nx)) for _ in range(3)]
    iux = iuy = None
    if init is not None:
        iux, iuy = _d(init[0]), _d(init[1])
    lib().oro_poc_grid(_p(a), _p(b), w, h, _p(xs), nx, _p(ys), ny, int(wy), int(wx), _p(iux), _p(iuy),
                       *[_p(o) for o in out])
    return out


def grid_shape(shape, cfg=None):
    pc, _ = _cfg(cfg)
    nx, ny = ctypes.c_int(), ctypes.c_int()
    lib().oro_grid_shape(int(shape[1]), int(shape[0]), pc, ctypes.byref(nx), ctypes.byref(ny))
    return ny.value, nx.value


def coarse_flow(I1, I2, cfg=None, init_dense=None):
    """poc.coarse_flow: dict(xs, ys, ux, uy, peak)."""
    a, b = _d(I1), _d(I2)
    h, w = a.shape
    ny, nx = grid_shape(a.shape, cfg)
    pc, _ = _cfg(cfg)
    xs, ys = np.empty(nx, np.int32), np.empty(ny, np.int32)
    out = [np.empty((ny, nx)) for _ in range(3)]
    iux = iuy = None
    if init_dense is not None:
        iux, iuy = _d(init_dense[0]), _d(init_dense[1])
    lib().oro_coarse_flow(_p(a), _p(b), w, h, _p(iux), _p(iuy), pc, _p(xs), _p(ys), *[_p(o) for o in out])
    return dict(xs=xs, ys=ys, ux=out[0], uy=out[1], peak=out[2])


def displacement_gradient(ux, uy, win):
    ux, uy = _d(ux), _d(uy)
    h, w = ux.shape
    out = [np.empty((h, w)) for _ in range(4)]
    lib().oro_displacement_gradient(_p(ux), _p(uy), w, h, int(win), *[_p(o) for o in out])
    return tuple(out)


def finish(ux, uy, conf, cfg=None, mask=None):
    """track._finish: (mx, my, strain dict)."""
    ux, uy, conf = _d(ux), _d(uy), _d(conf)
    h, w = ux.shape
    pc, _ = _cfg(cfg)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    out = [np.empty((h, w)) for _ in range(7)]
    lib().oro_finish(_p(ux), _p(uy), _p(conf), _p(m), w, h, pc, *[_p(o) for o in out])
    return out[0], out[1], dict(zip(("Exx", "Eyy", "Exy", "gmax", "vol"), out[2:]))


def track_pair(I1, I2, cfg=None, mask=None, init=None):
    """track.track_pair: dict(ux, uy, conf, Exx, Eyy, Exy, gmax, vol, raw_ux, raw_uy, valid, timing)."""
    a, b = _d(I1), _d(I2)
    h, w = a.shape
    pc, _ = _cfg(cfg)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    iux = iuy = None
    if init is not None:
        iux, iuy = _d(init[0]), _d(init[1])
    out = np.empty((10, h, w))
    timing = np.zeros(3)
    lib().oro_track_pair(_p(a), _p(b), w, h, _p(m), _p(iux), _p(iuy), pc, _p(out), _p(timing))
    names = ("ux", "uy", "conf", "Exx", "Eyy", "Exy", "gmax", "vol", "raw_ux", "raw_uy")
    r = {k: out[i] for i, k in enumerate(names)}
    r["valid"] = np.isfinite(r["ux"])
    r["timing"] = dict(coarse=timing[0], fine=timing[1], strain=timing[2])
    return r


# ---- temporal averaging front-end: the reference CLI's arithmetic (rust/crates/optflow-cli/src/tavg.rs), which
# follows python/optflow_ref/tavg.py except for its warp (the B-spline of interp::warp instead of scipy's
# map_coordinates; they agree away from the image border)

def _tavg_lstsq(xs, ys, v, sel):
    """v = c0 + c1 x + c2 y through the selected points, centred coordinates, Gaussian elimination with partial
    pivoting on the normal equations (tavg.rs:34-79); None on a pivot below 1e-12."""
    mx, my = xs[sel].mean(), ys[sel].mean()
    rows = np.stack([np.ones(sel.sum()), xs[sel] - mx, ys[sel] - my], axis=1)
    a = np.zeros((3, 4))
    for row, val in zip(rows, v[sel]):
        a[:, :3] += np.outer(row, row)
        a[:, 3] += row * val
    for c in range(3):
        p = c
        for i in range(c + 1, 3):
            if abs(a[i, c]) >= abs(a[p, c]):
                p = i
        if abs(a[p, c]) < 1e-12:
            return None
        a[[c, p]] = a[[p, c]]
        for i in range(c + 1, 3):
            f = a[i, c] / a[c, c]
            a[i, c:] -= f * a[c, c:]
    x = np.zeros(3)
    for i in (2, 1, 0):
        x[i] = (a[i, 3] - sum(a[i, j] * x[j] for j in range(i + 1, 3))) / a[i, i]
    return np.array([x[0] - x[1] * mx - x[2] * my, x[1], x[2]])


def tavg_fit_affine(xs, ys, ux, uy):
    """Robust affine through scattered displacements (tavg.rs:81-114): (cx, cy) or None."""
    xs, ys, ux, uy = (np.asarray(a, np.float64) for a in (xs, ys, ux, uy))
    sel = np.ones(len(xs), bool)
    coef = None
    for _ in range(4):
        if sel.sum() < 6:
            return None
        cx, cy = _tavg_lstsq(xs, ys, ux, sel), _tavg_lstsq(xs, ys, uy, sel)
        if cx is None or cy is None:
            return None
        coef = (cx, cy)
        r = np.hypot(cx[0] + cx[1] * xs + cx[2] * ys - ux, cy[0] + cy[1] * xs + cy[2] * ys - uy)
        mad = 1.4826 * np.median(r[sel])
        sel = r <= max(3.0 * mad, 0.05)
    return coef


def grid_sample(grid, x, y):
    """Bilinear interpolation of the grid field clamped to the grid (poc.rs:546-572)."""
    def frac(q, nodes):
        n = len(nodes)
        if n == 1:
            return np.zeros_like(q), np.zeros(q.shape, int), np.zeros(q.shape, int)
        step = float(nodes[1] - nodes[0])
        f = np.clip((q - nodes[0]) / step, 0.0, n - 1.0)
        i0 = np.minimum(np.floor(f).astype(int), n - 2)
        return f - i0, i0, np.minimum(i0 + 1, n - 1)
    tx, x0, x1 = frac(np.asarray(x, np.float64), grid["xs"])
    ty, y0, y1 = frac(np.asarray(y, np.float64), grid["ys"])
    out = []
    for a in (np.asarray(grid["ux"], np.float32).astype(np.float64), np.asarray(grid["uy"], np.float32).astype(np.float64)):
        out.append((1 - ty) * ((1 - tx) * a[y0, x0] + tx * a[y0, x1]) + ty * ((1 - tx) * a[y1, x0] + tx * a[y1, x1]))
    return out


def warp(img, ux, uy):
    """interp::warp (rust/crates/optflow-core/src/interp.rs:390-414): img at (x + ux, y + uy) by its cubic B-spline."""
    h, w = img.shape
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    c = bspline_coeffs(np.asarray(img, np.float32).astype(np.float64))
    return sample(c, xx + np.asarray(ux, np.float64), yy + np.asarray(uy, np.float64))


def align_to(centre, other, cfg=None, mask=None, model="affine"):
    """tavg::align_to (tavg.rs:116-161): `other` on the pixel grid of `centre`, or None."""
    h, w = centre.shape
    g = coarse_flow(centre, other, cfg)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    if model == "dense":
        ux, uy = grid_sample(g, xx, yy)
    else:
        Y, X = np.meshgrid(g["ys"], g["xs"], indexing="ij")
        ok = np.asarray(g["peak"], np.float32) > 0
        if mask is not None:
            ok &= np.asarray(mask, bool)[Y, X]
        if ok.sum() < 6:
            return None
        coef = tavg_fit_affine(X[ok], Y[ok], np.asarray(g["ux"], np.float32)[ok], np.asarray(g["uy"], np.float32)[ok])
        if coef is None:
            return None
        cx, cy = coef
        ux = cx[0] + cx[1] * xx + cx[2] * yy
        uy = cy[0] + cy[1] * xx + cy[2] * yy
    ux, uy = np.float32(ux).astype(np.float64), np.float32(uy).astype(np.float64)  # the CLI's float32 fields
    return np.float32(warp(other, ux, uy))


def average_window(frames, centre, align=False, cfg=None, mask=None, keep_unaligned=False, model="affine"):
    """tavg::average_window_with (tavg.rs:163-210): float32 mean (float64 sums: the others in order, then the
    centre) of the window."""
    c = np.asarray(frames[centre], np.float32)
    used = []
    for i, f in enumerate(frames):
        if i == centre:
            continue
        f = np.asarray(f, np.float32)
        if align:
            a = align_to(c, f, cfg, mask, model)
            if a is None:
                if not keep_unaligned:
                    continue
                a = f
            f = a
        used.append(f.astype(np.float64))
    if not used:
        return c.copy()
    s = used[0].copy()
    for u in used[1:]:
        s += u
    return np.float32((c.astype(np.float64) + s) / (len(used) + 1))


# ---------------------------------------------------------------- hybrid sequence gate
def _window_sum(a, r):
    """Sum over the (2r + 1)^2 window around every pixel, zero outside the image (hybrid.rs:69-108, the reference's
    uniform_filter(mode="constant") * size^2), by a summed-area table."""
    h, w = a.shape
    s = np.zeros((h + 1, w + 1))
    s[1:, 1:] = np.cumsum(np.cumsum(a, axis=0), axis=1)
    y0 = np.clip(np.arange(h) - r, 0, h)
    y1 = np.clip(np.arange(h) + r + 1, 0, h)
    x0 = np.clip(np.arange(w) - r, 0, w)
    x1 = np.clip(np.arange(w) + r + 1, 0, w)
    return (s[y1][:, x1] - s[y0][:, x1] - s[y1][:, x0] + s[y0][:, x0])


def local_affine_agreement(ux, uy, support, tx, ty, radius, min_support, tol):
    """_local_affine_agreement (python/optflow_ref/track.py:331-382; rust/crates/optflow-core/src/track/hybrid.rs:
    146-250): per pixel p the affine model u(q) = a + B (q - p), ridge 1e-3 r^2 on B, fitted by least squares to
    (ux, uy) of the support pixels in the window of half-size r = max(1, round(radius)); two passes, the second
    without the support pixels whose residual against their own first-pass model exceeds 3 tol. Returns (ok, n):
    ok = n + 0.5 >= min_support, n >= 3 and |(tx, ty) - a| <= tol; n = the support of the last pass."""
    h, w = ux.shape
    r = max(1, int(round(radius)))
    ridge = 1e-3 * r * r
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    support = np.asarray(support, bool)
    u0, v0 = np.where(support, ux, 0.0), np.where(support, uy, 0.0)
    sel = support.copy()
    for it in range(2):
        wt = sel.astype(np.float64)
        S = [_window_sum(wt * f, r) for f in (np.ones_like(xx), xx, yy, xx * xx, xx * yy, yy * yy)]
        s1, sx, sy, sxx, sxy, syy = S
        m = np.empty((h, w, 3, 3))
        m[..., 0, 0] = s1
        m[..., 0, 1] = m[..., 1, 0] = sx - xx * s1
        m[..., 0, 2] = m[..., 2, 0] = sy - yy * s1
        m[..., 1, 1] = sxx - 2 * xx * sx + xx * xx * s1 + ridge * s1
        m[..., 1, 2] = m[..., 2, 1] = sxy - xx * sy - yy * sx + xx * yy * s1
        m[..., 2, 2] = syy - 2 * yy * sy + yy * yy * s1 + ridge * s1
        fit = s1 >= 3
        m[~fit] = np.eye(3)
        a = []
        for comp in (u0, v0):
            su, sxu, syu = (_window_sum(wt * f * comp, r) for f in (np.ones_like(xx), xx, yy))
            rhs = np.stack([su, sxu - xx * su, syu - yy * su], axis=-1)
            rhs[~fit] = 0.0
            a.append(np.where(fit, np.linalg.solve(m, rhs[..., None])[..., 0, 0], np.nan))
        if it == 0:
            with np.errstate(invalid="ignore"):
                sel = support & (np.hypot(ux - a[0], uy - a[1]) <= 3 * tol)
    with np.errstate(invalid="ignore"):
        ok = (s1 + 0.5 >= min_support) & fit & (np.hypot(tx - a[0], ty - a[1]) <= tol)
    return ok, np.rint(s1).astype(np.int64)


# ---------------------------------------------------------------- frame front-end
_PIX_SCALE = {"gray8": 255.0, "rgb24": 255.0, "rgba32": 255.0, "gray16": 65535.0, "rgb48": 65535.0}


def to_gray(px, pixel, scale=1):
    """The CLI's grey levels of a frame, box-downscaled and rounded to float32 (rust/crates/optflow-cli/src/io.rs:
    44-52 luminance and lut8, 150-256 gray_from, 258-281 downscale; video.rs:290-300 rgb_to_gray): v / 255 or
    v / 65535, 0.299 R + 0.587 G + 0.114 B left to right, then per block the rows summed left to right and the
    row sums in order, / scale^2. Returns (out float32, grey float64 before the downscale)."""
    a = np.asarray(px)
    if pixel == "f32":
        g = a.astype(np.float32).astype(np.float64)
    else:
        f = a.astype(np.float64) / _PIX_SCALE[pixel]
        g = f if f.ndim == 2 else 0.299 * f[..., 0] + 0.587 * f[..., 1] + 0.114 * f[..., 2]
    if scale == 1:
        return g.astype(np.float32), g
    oh, ow = g.shape[0] // scale, g.shape[1] // scale
    b = g[:oh * scale, :ow * scale].reshape(oh, scale, ow, scale)
    total = np.zeros((oh, ow))
    for dy in range(scale):
        rs = np.zeros((oh, ow))
        for dx in range(scale):
            rs = rs + b[:, dy, :, dx]
        total = total + rs
    return (total / float(scale * scale)).astype(np.float32), g


def render(p, h, w, field=None, ss=4):
    """synth.render (python/optflow_ref/synth.py:150-190): the float64 speckle image of pattern p (cx, cy, r, a)
    deformed by field (an object with .ofc(), the struct of include/optflow_cuda_synth.h; None: the reference
    image), ss x ss subsamples per pixel."""
    arrs = [_d(v) for v in (p.cx, p.cy, p.r, p.a)]
    out = np.empty((h, w))
    f = field.ofc() if field is not None else None
    lib().oro_render(*[_p(a) for a in arrs], ctypes.c_size_t(arrs[0].size), int(w), int(h), int(ss),
                     ctypes.byref(f) if f is not None else None, _p(out))
    return out


def coarse_peaks(I1, I2, cfg=None, level=0, init_dense=None):
    """The integer POC peak of every grid point of pyramid level `level` of coarse_flow (level 0 = full size): the
    window offset round(d) plus the argmax of the last shifted correlation surface evaluated there, minus the half
    window (poc.py:50, 82-88), as an (ny, nx, 2) int array of (x, y); INT_MIN where no window was evaluated.
    None when the level does not exist."""
    a, b = _d(I1), _d(I2)
    h, w = a.shape
    pc, _ = _cfg(cfg)
    iux = iuy = None
    if init_dense is not None:
        iux, iuy = _d(init_dense[0]), _d(init_dense[1])
    cap = 2 * (h * w + 16)
    buf = np.empty(cap, np.int32)
    nx, ny = ctypes.c_int(), ctypes.c_int()
    n = lib().oro_coarse_peaks(_p(a), _p(b), w, h, _p(iux), _p(iuy), pc, int(level), _p(buf), ctypes.c_size_t(cap),
                               ctypes.byref(nx), ctypes.byref(ny))
    if n < 0:
        return None
    return buf[:2 * n].reshape(ny.value, nx.value, 2).copy()
