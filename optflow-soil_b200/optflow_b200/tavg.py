"""Temporal averaging front-end on the GPU: the reference's python/optflow_ref/tavg.py interface (align_to,
average_window) over the C ABI (ofc_align_to, ofc_average_window), with the reference CLI's arithmetic
(rust/crates/optflow-cli/src/tavg.rs: the robust affine fit in centred coordinates, float32 fields, the cubic
B-spline warp of interp::warp, the float64 mean)."""
import ctypes

import numpy as np

from ._abi import c_float_p, c_u8_p
from .api import _f32, _prep_cfg, _ptr, default_engine

_MODELS = {"affine": 0, "dense": 1}


def _model(cfg):
    m = getattr(cfg, "tavg_model", "affine")
    if m not in _MODELS:
        raise ValueError(f"tavg_model must be 'affine' or 'dense', got {m!r}")
    return _MODELS[m]


def _mask(mask, shape):
    if mask is None:
        return None
    m = np.ascontiguousarray(mask, dtype=bool)
    if m.shape != shape:
        raise ValueError(f"mask of shape {m.shape} for images of shape {shape}")
    return m.astype(np.uint8)


def align_to(centre, other, cfg=None, mask=None, engine=None):
    """tavg.align_to (python/optflow_ref/tavg.py:30-58): `other` resampled onto the pixel grid of `centre` by the
    motion of the coarse POC flow centre -> other (cfg.tavg_model: the robust affine fit inside `mask`, or the dense
    coarse flow), or None when no motion could be estimated."""
    eng = engine or default_engine()
    cfg, c = _prep_cfg(cfg)
    a = _f32(centre)
    h, w = a.shape
    b = _f32(other, (h, w))
    m = _mask(mask, (h, w))
    out = np.empty((h, w), np.float32)
    ok = ctypes.c_int(0)
    eng._call("ofc_align_to", _ptr(a, c_float_p), _ptr(b, c_float_p), w, h, _ptr(m, c_u8_p), _model(cfg),
              ctypes.byref(c), _ptr(out, c_float_p), ctypes.byref(ok))
    return out if ok.value else None


def average_window(frames, centre, align=False, cfg=None, mask=None, keep_unaligned=False, engine=None):
    """tavg.average_window (python/optflow_ref/tavg.py:61-74): the mean of `frames` (the window around
    frames[centre]); with align every other frame is first aligned to the centre (align_to), and one whose motion
    cannot be estimated is left out, or with keep_unaligned enters unaligned."""
    eng = engine or default_engine()
    cfg, c = _prep_cfg(cfg)
    fr = [_f32(f) for f in frames]
    if not fr:
        raise ValueError("no frames")
    h, w = fr[0].shape
    for f in fr:
        if f.shape != (h, w):
            raise ValueError("frames of different shapes")
    m = _mask(mask, (h, w))
    ptrs = (c_float_p * len(fr))(*[_ptr(f, c_float_p) for f in fr])
    out = np.empty((h, w), np.float32)
    used = ctypes.c_int(0)
    mode = (1 + _model(cfg)) if align else 0
    eng._call("ofc_average_window", ptrs, len(fr), int(centre), w, h, mode, _ptr(m, c_u8_p), int(bool(keep_unaligned)),
              ctypes.byref(c), _ptr(out, c_float_p), ctypes.byref(used))
    return out
