"""Frames in, results out: the CLI's frame front-end and output path over the C ABI.

to_gray (ofc_to_gray) is io.py's to_gray + downscale with the CLI's arithmetic (rust/crates/optflow-cli/src/io.rs:
44-52, 258-281: float64, the block's rows summed in order, rounded to float32). track_stream (ofc_track_stream) is
`optflow seq` on an iterable of frames: the engine pulls frame k + 1 into page-locked memory while it tracks frame k,
converts and downscales it on the GPU, and hands frame k's results over while it tracks frame k + 1; this generator
yields them as they come. save_result writes a result as io.py:203-233 does.
"""
import ctypes
import json
import os
import queue
import threading

import numpy as np

from . import _abi
from ._abi import OfcPairOut, c_float_p, c_u8_p
from .api import Result, _prep_cfg, _ptr, default_engine


def pixel_format(a):
    """The OFC_PIX_* name of an image array: uint8 / uint16 grey (H, W), uint8 RGB or RGBA (H, W, 3|4), uint16 RGB
    (H, W, 3), float grey (float64 is rounded to float32 first, the type the tracker works on)."""
    a = np.asarray(a)
    if a.ndim == 2:
        if a.dtype == np.uint8:
            return "gray8"
        if a.dtype == np.uint16:
            return "gray16"
        if a.dtype.kind == "f":
            return "f32"
    elif a.ndim == 3 and a.shape[2] in (3, 4):
        if a.dtype == np.uint8:
            return "rgb24" if a.shape[2] == 3 else "rgba32"
        if a.dtype == np.uint16 and a.shape[2] == 3:
            return "rgb48"
    raise ValueError(f"unsupported pixel type {a.dtype} of shape {a.shape}")


def _packed(a, fmt):
    dt = {"f32": np.float32, "gray8": np.uint8, "rgb24": np.uint8, "rgba32": np.uint8, "gray16": np.uint16,
          "rgb48": np.uint16}[fmt]
    return np.ascontiguousarray(a, dtype=dt)


def to_gray(a, scale=1, engine=None):
    """io.to_gray + io.downscale, rounded to float32 (the frames the CLI tracks): (H // scale, W // scale)."""
    eng = engine or default_engine()
    fmt = pixel_format(a)
    p = _packed(a, fmt)
    h, w = p.shape[:2]
    if scale < 1:
        raise ValueError(f"scale must be >= 1, got {scale}")
    out = np.empty((h // scale, w // scale), np.float32)
    eng._call("ofc_to_gray", p.ctypes.data_as(ctypes.c_void_p), _abi.OFC_PIX[fmt], w, h, int(scale),
              _ptr(out, c_float_p))
    return out


def _result(o, fb, info, shape):
    h, w = shape
    plane = lambda p: np.ctypeslib.as_array(p, (h, w)).copy()
    st = {"Exx": plane(o.exx), "Eyy": plane(o.eyy), "Exy": plane(o.exy), "gmax": plane(o.gmax), "vol": plane(o.vol)}
    timing = dict(coarse=o.timing[0], fine=o.timing[1], strain=o.timing[2], reference=int(info.reference),
                  mean_conf=float(info.mean_conf))
    r = Result(plane(o.ux), plane(o.uy), plane(o.conf), st, plane(o.raw_ux), plane(o.raw_uy), timing,
               np.ctypeslib.as_array(o.valid, (h, w)).astype(bool))
    if fb:
        r.fb = np.ctypeslib.as_array(fb, (h, w)).copy()
        r.timing.update(n_fb_max=int(info.n_fb_max), fallback_frac=float(info.fallback_frac),
                        fb_gate_rejected=float(info.fb_gate_rejected), reacquired=float(info.reacquired))
    return r


def track_stream(frames, cfg=None, mask=None, scale=1, start=0, stop=None, step=1, tavg=0, align=False,
                 align_mask=None, engine=None):
    """track.track_sequence over io.iter_frames of an iterable of decoded frames (any format of pixel_format, all of
    one shape; every frame of the video from index 0), all on the GPU: the frames start, start + step, ... < stop,
    each downscaled by `scale`; tavg = m > 0: each the mean of the downscaled frames i - m .. i + m (align: aligned to
    frame i with the affine model inside align_mask, on the downscaled grid; otherwise the windows the input's ends
    make one-sided with the dense model), kept on the device. mask: the tracking ROI on the downscaled grid;
    cfg.seq_mode chain or hybrid. Yields (k, Result) as the engine delivers them, while it tracks the next frame."""
    if step < 1:
        raise ValueError(f"step must be >= 1, got {step}")
    if start < 0:
        raise ValueError(f"start must be >= 0, got {start}")
    if tavg < 0:
        raise ValueError(f"tavg must be >= 0, got {tavg}")
    cfg, c = _prep_cfg(cfg)
    eng = engine or default_engine()
    it = iter(frames)
    try:
        first = np.asarray(next(it))
    except StopIteration:
        raise ValueError("no frames") from None
    fmt = pixel_format(first)
    h_in, w_in = first.shape[:2]
    if scale < 1:
        raise ValueError(f"scale must be >= 1, got {scale}")
    shape = (h_in // scale, w_in // scale)
    m = None
    if mask is not None:
        if np.shape(mask) != shape:
            raise ValueError(f"ROI mask shape {np.shape(mask)} differs from the frame shape {shape}")
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        if not m.any():
            raise ValueError("ROI mask is empty")
    am = None
    if align_mask is not None:
        if np.shape(align_mask) != shape:
            raise ValueError(f"align mask shape {np.shape(align_mask)} differs from the frame shape {shape}")
        am = np.ascontiguousarray(align_mask, dtype=np.uint8)
    nbytes = _packed(first, fmt).nbytes
    out_q = queue.Queue(maxsize=2)
    halt = threading.Event()
    state = {"first": first, "error": None, "pos": 0}  # pos: the index of the iterator's next frame

    def source(_user, k, dst):
        try:
            if halt.is_set():
                return 2
            while True:  # the engine asks for raw frame indices in increasing order; frames between are skipped
                if state["first"] is not None:
                    a, state["first"] = state["first"], None
                else:
                    a = next(it)
                state["pos"] += 1
                if state["pos"] - 1 == k:
                    break
            p = _packed(a, fmt)
            if p.nbytes != nbytes or p.shape[:2] != (h_in, w_in):
                raise ValueError(f"frame {k} has shape {np.shape(a)}, expected {first.shape}")
            ctypes.memmove(dst, p.ctypes.data, nbytes)
            return 0
        except StopIteration:
            return 1
        except Exception as e:  # noqa: BLE001 -- handed to the consumer after the engine returns
            state["error"] = e
            return 2

    def sink(_user, k, out, fb, info):
        if halt.is_set():
            return 1
        r = _result(ctypes.cast(out, ctypes.POINTER(OfcPairOut)).contents, fb, info.contents, shape)
        while not halt.is_set():
            try:
                out_q.put((int(k), r), timeout=0.1)
                return 0
            except queue.Full:
                continue
        return 1

    hy = _abi.OfcHybrid(int(cfg.fb_max), float(cfg.fb_radius), int(cfg.fb_min_support), float(cfg.fb_tol))
    src_fn, sink_fn = _abi.SOURCE_FN(source), _abi.SINK_FN(sink)
    s = _abi.OfcStream(_abi.OFC_PIX[fmt], w_in, h_in, int(scale), int(cfg.seq_mode == "hybrid"), hy,
                       float(cfg.ref_update_conf), src_fn, None, sink_fn, None, int(start), int(step),
                       -1 if stop is None else int(stop), int(tavg), int(bool(align)), _ptr(am, c_u8_p))
    done = object()

    def work():
        try:
            n = ctypes.c_int64(0)
            eng._call("ofc_track_stream", ctypes.byref(s), _ptr(m, c_u8_p), ctypes.byref(c), ctypes.byref(n))
        except Exception as e:  # noqa: BLE001
            if state["error"] is None and not halt.is_set():
                state["error"] = e
        finally:
            while True:
                try:
                    out_q.put(done, timeout=0.1)
                    break
                except queue.Full:
                    if halt.is_set():
                        break

    th = threading.Thread(target=work, name="ofc_track_stream", daemon=True)
    th.start()
    try:
        while True:
            item = out_q.get()
            if item is done:
                break
            yield item
    finally:
        halt.set()
        while th.is_alive():
            try:
                out_q.get(timeout=0.1)
            except queue.Empty:
                pass
        th.join()
    if state["error"] is not None:
        raise state["error"]


def save_result(out_dir, res, raw=False):
    """io.save_result (python/optflow_ref/io.py:203-233) without the crack outputs: ux, uy, conf, the strain fields
    (float32), valid (uint8), raw_ux / raw_uy with raw, fb of hybrid sequences, timing.json."""
    os.makedirs(out_dir, exist_ok=True)
    arrays = {"ux": res.ux, "uy": res.uy, "conf": res.conf}
    arrays.update({k: res.strain[k] for k in ("Exx", "Eyy", "Exy", "gmax", "vol")})
    if raw:
        arrays.update({"raw_ux": res.raw_ux, "raw_uy": res.raw_uy})
    for name, a in arrays.items():
        np.save(os.path.join(out_dir, f"{name}.npy"), np.ascontiguousarray(a, dtype="<f4"))
    np.save(os.path.join(out_dir, "valid.npy"), np.isfinite(res.ux).astype(np.uint8))
    if res.fb is not None:
        np.save(os.path.join(out_dir, "fb.npy"), np.ascontiguousarray(res.fb, dtype="<i4"))
    with open(os.path.join(out_dir, "timing.json"), "w") as f:
        json.dump(res.timing, f, indent=2)


def iter_frames(frames, start=0, stop=None, step=1, scale=1, tavg=0, align=False, cfg=None, mask_fn=None,
                engine=None):
    """io.iter_frames (python/optflow_ref/io.py:100-153) over an iterable of decoded frames (every frame of the
    video or image list, from index 0): frames start, start + step, ... < stop, each turned grey and downscaled on
    the GPU (to_gray). tavg = m > 0: each is the mean of frames i - m .. i + m (clipped to the input) after the
    downscale (tavg.average_window on the GPU); a window that is one-sided because the input ends has its
    neighbours aligned with the dense model and keep_unaligned, unless `align` aligns every window (affine model of
    cfg, mask_fn(shape) the ROI of the fit)."""
    import dataclasses

    from .config import Config
    from .tavg import average_window
    if step < 1:
        raise ValueError(f"step must be >= 1, got {step}")
    if start < 0:
        raise ValueError(f"start must be >= 0, got {start}")
    if tavg < 0:
        raise ValueError(f"tavg must be >= 0, got {tavg}")
    m = int(tavg)
    lo_read = max(0, start - m)
    hi_read = None if stop is None else stop + m
    if not m:
        for i, f in enumerate(frames):
            if stop is not None and i >= stop:
                break
            if i >= start and (i - start) % step == 0:
                yield to_gray(f, scale, engine=engine)
        return
    cfg = cfg or Config()
    edge_cfg = dataclasses.replace(cfg, tavg_model="dense")
    buf = {}
    nxt, last = start, -1

    def emit(s):
        lo, hi = max(0, s - m), min(s + m, last)
        fr = [buf[i] for i in range(lo, hi + 1)]
        if not align and s - lo != hi - s and min(fr[0].shape) >= edge_cfg.poc_win:
            return average_window(fr, s - lo, True, edge_cfg, None, keep_unaligned=True, engine=engine)
        return average_window(fr, s - lo, align, cfg, mask_fn(fr[0].shape) if align and mask_fn else None,
                              engine=engine)

    def due(i_ready):
        return (stop is None or nxt < stop) and nxt <= i_ready

    for i, f in enumerate(frames):
        if i < lo_read:
            continue
        if hi_read is not None and i >= hi_read:
            break
        buf[i], last = to_gray(f, scale, engine=engine), i
        while due(i - m):
            yield emit(nxt)
            nxt += step
            for j in [j for j in buf if j < nxt - m]:
                del buf[j]
    while due(last):
        yield emit(nxt)
        nxt += step
