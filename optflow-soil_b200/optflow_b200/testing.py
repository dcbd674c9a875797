"""Single-stage entry points of the CUDA engine (include/optflow_cuda_testing.h), for the parity tests."""
import ctypes

import numpy as np

from ._abi import c_double_p, c_float_p, c_i32_p, c_u8_p
from .api import _f32, _ptr, default_engine
from .config import Config


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def fft_lines(data, inverse=False, engine=None):
    """Row-wise FFT of a 2-D complex array (numpy fft; inverse: L * numpy ifft)."""
    eng = engine or default_engine()
    a = np.ascontiguousarray(data, dtype=np.complex64).copy()
    lines, L = a.shape
    eng._call("ofc_test_fft_lines", a.ctypes.data_as(c_float_p), lines, L, int(inverse))
    return a


def reference_phase(I1, cfg=None, engine=None):
    eng = engine or default_engine()
    cfg = cfg or Config()
    c = cfg.to_ofc()
    a = _f32(I1)
    h, w = a.shape
    F = cfg.n_filters()
    out = [np.empty((F, h, w), np.float32) for _ in range(5)]
    eng._call("ofc_test_reference_phase", _ptr(a, c_float_p), w, h, ctypes.byref(c), *[_ptr(o, c_float_p) for o in out])
    re, im, gx, gy, amp = out
    return [(re[k] + 1j * im[k], gx[k], gy[k], amp[k]) for k in range(F)]


def responses(img, cfg=None, engine=None):
    eng = engine or default_engine()
    cfg = cfg or Config()
    c = cfg.to_ofc()
    a = _f32(img)
    h, w = a.shape
    F = cfg.n_filters()
    out = np.empty((F, h + 64, w + 64), np.complex64)
    eng._call("ofc_test_responses", _ptr(a, c_float_p), w, h, ctypes.byref(c), out.ctypes.data_as(c_float_p))
    return out


def local_solve(sums, ux, uy, cfg=None, engine=None):
    eng = engine or default_engine()
    cfg = cfg or Config()
    c = cfg.to_ofc()
    s = _d(np.stack(sums))
    ux, uy = _d(ux), _d(uy)
    h, w = ux.shape
    out = [np.empty((h, w)) for _ in range(4)]
    slope = np.empty((4, h, w))
    eng._call("ofc_test_local_solve", _ptr(s, c_double_p), _ptr(ux, c_double_p), _ptr(uy, c_double_p), w, h,
              ctypes.byref(c), *[_ptr(o, c_double_p) for o in out], _ptr(slope, c_double_p))
    return (*out, np.moveaxis(slope, 0, -1))


def median(v, engine=None):
    eng = engine or default_engine()
    a = _d(v).ravel()
    out = ctypes.c_double()
    eng._call("ofc_test_median", _ptr(a, c_double_p), a.size, ctypes.byref(out))
    return out.value


def large_components(b, min_area, engine=None):
    eng = engine or default_engine()
    a = np.ascontiguousarray(b, dtype=np.uint8)
    h, w = a.shape
    out = np.empty_like(a)
    eng._call("ofc_test_large_components", _ptr(a, c_u8_p), w, h, ctypes.c_double(min_area), _ptr(out, c_u8_p))
    return out.astype(bool)


def poc_peaks(I1, I2, cfg=None, level=0, engine=None):
    """The integer POC peaks of pyramid level `level` of coarse_flow (ofc_test_poc_peaks): (ny, nx, 2) int32 of
    (x, y), INT_MIN where no window was evaluated."""
    eng = engine or default_engine()
    a, b = _f32(I1), _f32(I2)
    h, w = a.shape
    c = (cfg or Config()).to_ofc()
    cap = 2 * (h * w + 16)
    buf = np.empty(cap, np.int32)
    nx, ny = ctypes.c_int32(), ctypes.c_int32()
    eng._call("ofc_test_poc_peaks", _ptr(a, c_float_p), _ptr(b, c_float_p), w, h, ctypes.byref(c), int(level),
              _ptr(buf, c_i32_p), cap, ctypes.byref(nx), ctypes.byref(ny))
    return buf[:2 * nx.value * ny.value].reshape(ny.value, nx.value, 2).copy()


def prewarp_fill(low, ux, uy, slope, radius, engine=None):
    """slope: (h, w, 4) as in phaseflow.Flow.slope."""
    eng = engine or default_engine()
    lo = np.ascontiguousarray(low, dtype=np.uint8)
    h, w = lo.shape
    ux, uy = _d(ux), _d(uy)
    sl = _d(np.moveaxis(np.asarray(slope), -1, 0))
    ox, oy = np.empty((h, w)), np.empty((h, w))
    eng._call("ofc_test_prewarp_fill", _ptr(lo, c_u8_p), _ptr(ux, c_double_p), _ptr(uy, c_double_p),
              _ptr(sl, c_double_p), w, h, ctypes.c_double(radius), _ptr(ox, c_double_p), _ptr(oy, c_double_p))
    return ox, oy


def first_sums(I1, I2, ux, uy, cfg=None, engine=None):
    """The seven per-pixel sums of refine's first inner iteration from the start field (ux, uy)."""
    eng = engine or default_engine()
    cfg = cfg or Config()
    c = cfg.to_ofc()
    a, b = _f32(I1), _f32(I2)
    h, w = a.shape
    ux, uy = _d(ux), _d(uy)
    out = np.empty((7, h, w))
    eng._call("ofc_test_first_sums", _ptr(a, c_float_p), _ptr(b, c_float_p), w, h, _ptr(ux, c_double_p),
              _ptr(uy, c_double_p), ctypes.byref(c), _ptr(out, c_double_p))
    return out


def accumulate(I1, I2, ux, uy, mode=1, cfg=None, engine=None):
    """first_sums with the accumulate kernel chosen: mode 0 the gather kernel, mode 1 the TMA-staged kernel.
    Returns (sums (7, h, w), stage waits that gave up)."""
    eng = engine or default_engine()
    cfg = cfg or Config()
    c = cfg.to_ofc()
    a, b = _f32(I1), _f32(I2)
    h, w = a.shape
    ux, uy = _d(ux), _d(uy)
    out = np.empty((7, h, w))
    tmo = ctypes.c_uint32(0)
    eng._call("ofc_test_accumulate", _ptr(a, c_float_p), _ptr(b, c_float_p), w, h, _ptr(ux, c_double_p),
              _ptr(uy, c_double_p), ctypes.byref(c), int(mode), _ptr(out, c_double_p), ctypes.byref(tmo))
    return out, tmo.value


def warp(c2, sx, sy, shift=(0, 0), mode=1, engine=None):
    """The B-spline warp of coefficient plane c2 (h2 x w2 float32) at (x + shift_x + sx, y + shift_y + sy) for fields
    sx, sy (h x w float64), by the gather kernel (mode 0) or the TMA-staged kernel (mode 1): (out float32 h x w,
    timed-out tile waits)."""
    eng = engine or default_engine()
    c = _f32(c2)
    h2, w2 = c.shape
    fx, fy = _d(sx), _d(sy)
    h, w = fx.shape
    out = np.empty((h, w), np.float32)
    tmo = ctypes.c_uint32(0)
    eng._call("ofc_test_warp", _ptr(c, c_float_p), w2, h2, _ptr(fx, c_double_p), _ptr(fy, c_double_p),
              int(shift[0]), int(shift[1]), w, h, int(mode), _ptr(out, c_float_p), ctypes.byref(tmo))
    return out, tmo.value


def atan2(y, x, engine=None):
    """The accumulate's float32 atan2 and CUDA's atan2f on the device for float32 arrays y, x: (mine, cuda)."""
    eng = engine or default_engine()
    yy = np.ascontiguousarray(y, dtype=np.float32).ravel()
    xx = np.ascontiguousarray(x, dtype=np.float32).ravel()
    mine = np.empty_like(yy)
    cuda = np.empty_like(yy)
    eng._call("ofc_test_atan2", _ptr(yy, c_float_p), _ptr(xx, c_float_p), yy.size, _ptr(mine, c_float_p),
              _ptr(cuda, c_float_p))
    return mine.reshape(np.shape(y)), cuda.reshape(np.shape(y))
