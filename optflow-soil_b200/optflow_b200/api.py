"""The reference's Python API (python/optflow_ref) over the CUDA engine's C ABI.

``track_pair``, ``refine``, ``coarse_flow``, ``displacement_gradient``, ``strain_fields`` and the
``_finish`` step keep the reference's names, argument meaning and error behaviour (ValueError for bad
input, as the reference raises), so tests written against the reference read the same here. Every
call runs on the GPU through ``liboptflow_cuda.so``; there is no CPU path.
"""
import ctypes
import threading
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import EngineError, OfcPairOut, c_double_p, c_float_p, c_i32_p, c_u8_p
from .config import Config

_ERRLEN = 1024


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


def _ptr(a, typ):
    return None if a is None else a.ctypes.data_as(typ)


class Engine:
    """An engine on one CUDA device (GpuEngine of rust/crates/optflow-gpu/src/engine.rs:94-103).

    Holds the device context, plans and pooled buffers between calls until ``release_caches``.
    """

    def __init__(self, device=0, lanes=1):
        self.lib = _abi.load()
        from .fftplan import install
        install()
        err = ctypes.create_string_buffer(_ERRLEN)
        h = self.lib.ofc_create(int(device), int(lanes), err, _ERRLEN)
        if not h:
            raise EngineError(_abi.OFC_ERR_DEVICE if hasattr(_abi, "OFC_ERR_DEVICE") else 2,
                              err.value.decode() or "ofc_create failed")
        self.handle = ctypes.c_void_p(h)
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            self.lib.ofc_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call(self, name, *args):
        err = ctypes.create_string_buffer(_ERRLEN)
        st = getattr(self.lib, name)(self.handle, *args, err, _ERRLEN)
        if st != 0:
            msg = err.value.decode()
            if st == 1:
                raise ValueError(msg)
            raise EngineError(st, msg)

    @property
    def lanes(self):
        return self.lib.ofc_lanes(self.handle)

    def set_coarse_net(self, params=None, tile=256, max_low_share=0.25):
        """Pair calls without a start field start from the learned coarse proposal (include/optflow_cuda_net.h):
        params = the network's float32 parameters ("default": the trained set shipped with the package); None: back
        to the POC coarse stage. Tiles of tile x tile px whose refined result has more than max_low_share
        low-confidence pixels fall back to POC."""
        if isinstance(params, str) and params == "default":
            from .net import load_weights
            params = load_weights()
        if params is None:
            self._call("ofc_set_coarse_net", None, 0, int(tile), ctypes.c_double(max_low_share))
            return
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._call("ofc_set_coarse_net", p.ctypes.data_as(c_float_p), p.size, int(tile), ctypes.c_double(max_low_share))

    def coarse_net_stats(self):
        """Counters of the learned proposal: pairs, tiles judged, tiles failed, pairs that fell back to POC."""
        out = (ctypes.c_uint64 * 4)()
        self.lib.ofc_coarse_net_stats(self.handle, out)
        return dict(pairs=out[0], tiles=out[1], failed_tiles=out[2], fallback_pairs=out[3])

    def kernel_launches(self):
        return int(self.lib.ofc_kernel_launches(self.handle))

    def check_window(self, w, h, cfg=None):
        c = (cfg or Config()).to_ofc()
        self._call("ofc_check_window", ctypes.c_size_t(w), ctypes.c_size_t(h), ctypes.byref(c))

    def release_caches(self):
        self.lib.ofc_release_caches(self.handle)


_default = {}
_lock = threading.Lock()


def default_engine(device=0):
    """The module's engine on `device`, created on first use with two lanes: a frame source (iter_frames) may then
    call the engine while a streamed sequence (track_stream) holds the other lane."""
    with _lock:
        if device not in _default:
            _default[device] = Engine(device, lanes=2)
        return _default[device]


@dataclass
class Flow:
    """phaseflow.Flow (python/optflow_ref/phaseflow.py:53-60) without the crack bookkeeping."""
    ux: np.ndarray
    uy: np.ndarray
    conf: np.ndarray
    resid: np.ndarray
    low: np.ndarray = None


@dataclass
class Grid:
    """poc.Grid (python/optflow_ref/poc.py:9-15)."""
    xs: np.ndarray
    ys: np.ndarray
    ux: np.ndarray
    uy: np.ndarray
    peak: np.ndarray


@dataclass
class Result:
    """track.Result (python/optflow_ref/track.py:15-31) of one pair."""
    ux: np.ndarray
    uy: np.ndarray
    conf: np.ndarray
    strain: dict
    raw_ux: np.ndarray
    raw_uy: np.ndarray
    timing: dict = field(default_factory=dict)
    valid: np.ndarray = None
    fb: np.ndarray = None  # hybrid sequences only: frames each pixel has been carried by the adjacent leg


def _prep_cfg(cfg):
    cfg = cfg or Config()
    cfg.validate()
    return cfg, cfg.to_ofc()


def refine_raw(I1, I2, ux, uy, cfg=None, shift=(0, 0), engine=None):
    """FineEngine::refine_raw (rust/crates/optflow-core/src/engine.rs:32-40): dict of f64 planes
    ux, uy, energy, resid of the window I1 (I2 any part of the second image placed at `shift`)."""
    eng = engine or default_engine()
    cfg, c = _prep_cfg(cfg)
    a = _f32(I1)
    h, w = a.shape
    b = _f32(I2)
    u, v = _f32(ux, (h, w)), _f32(uy, (h, w))
    out = [np.empty((h, w), np.float64) for _ in range(4)]
    eng._call("ofc_refine_raw", _ptr(a, c_float_p), w, h, _ptr(b, c_float_p), b.shape[1], b.shape[0],
              ctypes.c_int64(shift[0]), ctypes.c_int64(shift[1]), _ptr(u, c_float_p), _ptr(v, c_float_p),
              ctypes.byref(c), *[_ptr(o, c_double_p) for o in out])
    return dict(zip(("ux", "uy", "energy", "resid"), out))


def refine_batch(windows, cfg=None, engine=None):
    """The refine_raw calls of a tiling driver's windows in one call (the tile loop of
    rust/crates/optflow-core/src/tile.rs:420-472): windows is a sequence of (I1, I2, ux, uy, shift);
    returns one refine_raw result dict per window, bit-identical to separate refine_raw calls."""
    eng = engine or default_engine()
    cfg, c = _prep_cfg(cfg)
    keep, outs = [], []
    arr = (_abi.OfcWindow * max(1, len(windows)))()
    for k, (I1, I2, ux, uy, shift) in enumerate(windows):
        a = _f32(I1)
        h, w = a.shape
        b = _f32(I2)
        u, v = _f32(ux, (h, w)), _f32(uy, (h, w))
        out = [np.empty((h, w), np.float64) for _ in range(4)]
        keep += [a, b, u, v]
        outs.append(out)
        arr[k] = _abi.OfcWindow(_ptr(a, c_float_p), w, h, _ptr(b, c_float_p), b.shape[1], b.shape[0], int(shift[0]),
                                int(shift[1]), _ptr(u, c_float_p), _ptr(v, c_float_p),
                                *[_ptr(o, c_double_p) for o in out])
    eng._call("ofc_refine_batch", ctypes.cast(arr, ctypes.c_void_p), len(windows), ctypes.byref(c))
    return [dict(zip(("ux", "uy", "energy", "resid"), out)) for out in outs]


def refine(I1, I2, ux, uy, cfg=None, engine=None) -> Flow:
    """phaseflow.refine (python/optflow_ref/phaseflow.py:427-511)."""
    eng = engine or default_engine()
    cfg, c = _prep_cfg(cfg)
    a = _f32(I1)
    h, w = a.shape
    b = _f32(I2, (h, w))
    u, v = _f32(ux, (h, w)), _f32(uy, (h, w))
    out = [np.empty((h, w), np.float32) for _ in range(4)]
    low = np.empty((h, w), np.uint8)
    eng._call("ofc_refine", _ptr(a, c_float_p), _ptr(b, c_float_p), w, h, _ptr(u, c_float_p), _ptr(v, c_float_p),
              ctypes.byref(c), *[_ptr(o, c_float_p) for o in out], _ptr(low, c_u8_p))
    return Flow(out[0], out[1], out[2], out[3], low.astype(bool))


def coarse_flow(I1, I2, cfg=None, init_dense=None, engine=None) -> Grid:
    """poc.coarse_flow (python/optflow_ref/poc.py:216-239)."""
    eng = engine or default_engine()
    cfg, c = _prep_cfg(cfg)
    a = _f32(I1)
    h, w = a.shape
    b = _f32(I2, (h, w))
    nx, ny = ctypes.c_size_t(), ctypes.c_size_t()
    if eng.lib.ofc_grid_shape(w, h, ctypes.byref(c), ctypes.byref(nx), ctypes.byref(ny)) != 0:
        raise ValueError(f"image {w}x{h} too small for poc_win {cfg.poc_win}")
    nx, ny = nx.value, ny.value
    xs, ys = np.empty(nx, np.int32), np.empty(ny, np.int32)
    gu, gv, gp = (np.empty((ny, nx), np.float32) for _ in range(3))
    iu = iv = None
    if init_dense is not None:
        iu, iv = _f32(init_dense[0], (h, w)), _f32(init_dense[1], (h, w))
    eng._call("ofc_coarse_flow", _ptr(a, c_float_p), _ptr(b, c_float_p), w, h, _ptr(iu, c_float_p),
              _ptr(iv, c_float_p), ctypes.byref(c), _ptr(xs, c_i32_p), _ptr(ys, c_i32_p), _ptr(gu, c_float_p),
              _ptr(gv, c_float_p), _ptr(gp, c_float_p))
    return Grid(xs, ys, gu, gv, gp)


def displacement_gradient(ux, uy, win, engine=None):
    """strain.displacement_gradient (python/optflow_ref/strain.py:61-97): (dudx, dudy, dvdx, dvdy)."""
    return _strain(ux, uy, win, engine)[:4]


def _strain(ux, uy, win, engine=None):
    eng = engine or default_engine()
    u = _f32(ux)
    h, w = u.shape
    v = _f32(uy, (h, w))
    out = [np.empty((h, w), np.float32) for _ in range(9)]
    eng._call("ofc_strain", _ptr(u, c_float_p), _ptr(v, c_float_p), w, h, int(win),
              *[_ptr(o, c_float_p) for o in out])
    return out


def strain_fields(dudx, dudy, dvdx, dvdy):
    """strain.strain_fields (python/optflow_ref/strain.py:100-112): host arithmetic on four maps."""
    exx = dudx + 0.5 * (dudx**2 + dvdx**2)
    eyy = dvdy + 0.5 * (dudy**2 + dvdy**2)
    exy = 0.5 * (dudy + dvdx) + 0.5 * (dudx * dudy + dvdx * dvdy)
    return {"Exx": exx, "Eyy": eyy, "Exy": exy, "exx": dudx, "eyy": dvdy, "exy": 0.5 * (dudy + dvdx),
            "gmax": 2.0 * np.sqrt(((exx - eyy) / 2) ** 2 + exy**2),
            "vol": (1 + dudx) * (1 + dvdy) - dudy * dvdx - 1.0}


def _pair_out(h, w):
    arrs = {k: np.empty((h, w), np.uint8 if k == "valid" else np.float32) for k in _abi.PAIR_FIELDS}
    o = OfcPairOut()
    for k, a in arrs.items():
        setattr(o, k, _ptr(a, c_u8_p if k == "valid" else c_float_p))
    return o, arrs


def _result(o, arrs):
    st = {"Exx": arrs["exx"], "Eyy": arrs["eyy"], "Exy": arrs["exy"], "gmax": arrs["gmax"], "vol": arrs["vol"]}
    timing = dict(coarse=o.timing[0], fine=o.timing[1], strain=o.timing[2])
    return Result(arrs["ux"], arrs["uy"], arrs["conf"], st, arrs["raw_ux"], arrs["raw_uy"], timing,
                  arrs["valid"].astype(bool))


def track_pairs(items, cfg=None, engine=None):
    """track_pair over many independent pairs of any sizes in one ofc_track_pairs call: items are (I1, I2),
    (I1, I2, mask) or (I1, I2, mask, init) tuples; returns the list of Results, each equal to track_pair's. The
    pairs overlap on the engine's worker lanes."""
    cfg, c = _prep_cfg(cfg)
    eng = engine or default_engine()
    items = list(items)
    ins = (_abi.OfcPairIn * max(len(items), 1))()
    outs = (OfcPairOut * max(len(items), 1))()
    keep, arrs = [], []
    for i, it in enumerate(items):
        I1, I2 = it[0], it[1]
        mask = it[2] if len(it) > 2 else None
        init = it[3] if len(it) > 3 else None
        a = _f32(I1)
        h, w = a.shape
        b = _f32(I2, (h, w))
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
        if m is not None and m.shape != (h, w):
            raise ValueError(f"pair {i}: ROI mask shape {m.shape} differs from the image shape {(h, w)}")
        u = v = None
        if init is not None:
            u, v = _f32(init[0], (h, w)), _f32(init[1], (h, w))
        ins[i] = _abi.OfcPairIn(_ptr(a, c_float_p), _ptr(b, c_float_p), w, h, _ptr(m, c_u8_p), _ptr(u, c_float_p),
                                _ptr(v, c_float_p))
        keep.append((a, b, m, u, v))
        o, arr = _pair_out(h, w)
        outs[i] = o
        arrs.append(arr)
    eng._call("ofc_track_pairs", ins, len(items), ctypes.byref(c), outs)
    return [_result(outs[i], arrs[i]) for i in range(len(items))]


def finish(ux, uy, conf, cfg=None, mask=None, engine=None) -> Result:
    """track._finish (python/optflow_ref/track.py:56-108) without the crack options."""
    eng = engine or default_engine()
    cfg, c = _prep_cfg(cfg)
    u = _f32(ux)
    h, w = u.shape
    v, cf = _f32(uy, (h, w)), _f32(conf, (h, w))
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    o, arrs = _pair_out(h, w)
    eng._call("ofc_finish", _ptr(u, c_float_p), _ptr(v, c_float_p), _ptr(cf, c_float_p), _ptr(m, c_u8_p), w, h,
              ctypes.byref(c), ctypes.byref(o))
    return _result(o, arrs)


def track_pair(I1, I2, cfg=None, mask=None, init=None, engine=None) -> Result:
    """track.track_pair (python/optflow_ref/track.py:115-146): the displacement of I1's pixels into I2."""
    I1 = np.asarray(I1)
    I2 = np.asarray(I2)
    if I1.shape != I2.shape:
        raise ValueError(f"image sizes differ: {I1.shape} vs {I2.shape}")
    if mask is not None and np.shape(mask) != I1.shape:
        raise ValueError(f"ROI mask shape {np.shape(mask)} differs from the image shape {I1.shape}")
    if mask is not None and not np.any(mask):
        raise ValueError("ROI mask is empty")
    cfg, c = _prep_cfg(cfg)
    if min(I1.shape) < cfg.poc_win:
        raise ValueError(f"image smaller than poc_win ({cfg.poc_win}): {I1.shape}")
    eng = engine or default_engine()
    a, b = _f32(I1), _f32(I2)
    h, w = a.shape
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    iu = iv = None
    if init is not None:
        iu, iv = _f32(init[0], (h, w)), _f32(init[1], (h, w))
    o, arrs = _pair_out(h, w)
    eng._call("ofc_track_pair", _ptr(a, c_float_p), _ptr(b, c_float_p), w, h, _ptr(m, c_u8_p),
              _ptr(iu, c_float_p), _ptr(iv, c_float_p), ctypes.byref(c), ctypes.byref(o))
    return _result(o, arrs)


def _check_frames(fr, cfg, mask):
    if not fr:
        raise ValueError("no frames")
    h, w = fr[0].shape
    for k, f in enumerate(fr):
        if f.shape != fr[0].shape:
            raise ValueError(f"frame {k} has shape {f.shape}, expected {fr[0].shape}")
    if mask is not None and np.shape(mask) != fr[0].shape:
        raise ValueError(f"ROI mask shape {np.shape(mask)} differs from the frame shape {fr[0].shape}")
    if mask is not None and not np.any(mask):
        raise ValueError("ROI mask is empty")
    if len(fr) > 1 and min(h, w) < cfg.poc_win:
        raise ValueError(f"image smaller than poc_win ({cfg.poc_win}): {fr[0].shape}")
    return h, w


def track_sequence(frames, cfg=None, mask=None, engine=None):
    """track.track_sequence (python/optflow_ref/track.py:260-315; rust/crates/optflow-core/src/track.rs:1030-1245):
    yields (k, Result) with the displacement from frame 0 to frame k, k = 1, 2, ...; Result.timing adds the reference
    index and the leg's mean confidence. The frames are tracked in one ofc_track_sequence call (all of them are read
    first); seq_mode "hybrid" goes to track_sequence_hybrid."""
    cfg, c = _prep_cfg(cfg)
    fr = [np.asarray(f) for f in frames]
    if not fr:
        raise ValueError("no frames")
    if cfg.seq_mode == "hybrid":
        yield from track_sequence_hybrid(fr, cfg, mask, engine=engine)
        return
    h, w = _check_frames(fr, cfg, mask)
    eng = engine or default_engine()
    f32 = [_f32(f) for f in fr]
    ptrs = (c_float_p * len(f32))(*[_ptr(f, c_float_p) for f in f32])
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    nk = max(len(fr) - 1, 1)
    outs = (OfcPairOut * nk)()
    arrs = []
    for k in range(len(fr) - 1):
        o, a = _pair_out(h, w)
        outs[k] = o
        arrs.append(a)
    ref = np.zeros(nk, np.int32)
    mean = np.zeros(nk)
    eng._call("ofc_track_sequence", ptrs, len(fr), w, h, _ptr(m, c_u8_p), ctypes.byref(c), float(cfg.ref_update_conf),
              outs, _ptr(ref, _abi.c_i32_p), _ptr(mean, c_double_p))
    for k in range(1, len(fr)):
        r = _result(outs[k - 1], arrs[k - 1])
        r.timing.update(reference=int(ref[k - 1]), mean_conf=float(mean[k - 1]))
        yield k, r


def track_sequence_hybrid(frames, cfg=None, mask=None, ref_update_conf=None, legs=None, engine=None):
    """track.track_sequence with seq_mode "hybrid" (python/optflow_ref/track.py:385-503; rust/crates/optflow-core/
    src/track/hybrid.rs) over ofc_track_sequence_hybrid: yields (k, Result) with Result.fb (the fallback counters)
    and the timing keys reference, mean_conf, n_fb_max, fallback_frac, fb_gate_rejected, reacquired.

    ref_update_conf: one threshold per frame k = 1..n-1 (default cfg.ref_update_conf for all; the reference reads the
    key anew at every frame). legs: a scripted leg source legs(i, j, init) -> (raw_ux, raw_uy, conf) that replaces
    the engine's pair tracking of the leg frames[i] -> frames[j] (init: None or the (ux, uy) start), as the
    reference's tests replace track_pair (python/tests/test_hybrid.py:38-52)."""
    cfg, c = _prep_cfg(cfg)
    fr = [np.asarray(f) for f in frames]
    h, w = _check_frames(fr, cfg, mask)
    nk = max(len(fr) - 1, 1)
    ruc = np.full(nk, float(cfg.ref_update_conf)) if ref_update_conf is None else \
        np.ascontiguousarray(ref_update_conf, dtype=np.float64)
    if ruc.shape != (nk,):
        raise ValueError(f"ref_update_conf needs one value per frame after the first ({nk})")
    eng = engine or default_engine()
    f32 = [_f32(f) for f in fr]
    ptrs = (c_float_p * len(f32))(*[_ptr(f, c_float_p) for f in f32])
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    outs = (OfcPairOut * nk)()
    arrs = []
    for k in range(len(fr) - 1):
        o, a = _pair_out(h, w)
        outs[k] = o
        arrs.append(a)
    fb = np.zeros((nk, h, w), np.int32)
    info = (_abi.OfcHybridFrame * nk)()
    hy = _abi.OfcHybrid(int(cfg.fb_max), float(cfg.fb_radius), int(cfg.fb_min_support), float(cfg.fb_tol))
    failure = []

    def leg(_user, i, j, iu, iv, rx, ry, rc):
        try:
            init = None
            if iu:
                init = (np.ctypeslib.as_array(iu, (h, w)).copy(), np.ctypeslib.as_array(iv, (h, w)).copy())
            out = legs(int(i), int(j), init)
            for dst, src in zip((rx, ry, rc), out):
                np.ctypeslib.as_array(dst, (h, w))[...] = np.broadcast_to(np.asarray(src, np.float32), (h, w))
            return 0
        except Exception as e:  # noqa: BLE001 -- handed back to the caller after the engine returns
            failure.append(e)
            return 1

    fn = _abi.LEG_FN(leg) if legs is not None else _abi.LEG_FN()
    try:
        eng._call("ofc_track_sequence_hybrid", ptrs, len(fr), w, h, _ptr(m, c_u8_p), ctypes.byref(c),
                  _ptr(ruc, c_double_p), ctypes.byref(hy), outs, _ptr(fb, _abi.c_i32_p), info, fn, None)
    except ValueError:
        if failure:
            raise failure[0]
        raise
    for k in range(1, len(fr)):
        r = _result(outs[k - 1], arrs[k - 1])
        f = info[k - 1]
        r.fb = fb[k - 1]
        r.timing.update(reference=int(f.reference), mean_conf=float(f.mean_conf), n_fb_max=int(f.n_fb_max),
                        fallback_frac=float(f.fallback_frac), fb_gate_rejected=float(f.fb_gate_rejected),
                        reacquired=float(f.reacquired))
        yield k, r


def local_affine_agreement(ux, uy, support, tx, ty, radius, min_support, tol, engine=None):
    """track._local_affine_agreement (python/optflow_ref/track.py:331-382) over ofc_local_affine_agreement: returns
    (ok, n), ok = the robust local affine model of (ux, uy) on `support` predicts (tx, ty) within tol with at least
    min_support pixels in the window, n = the number of them."""
    eng = engine or default_engine()
    a = np.ascontiguousarray(ux, dtype=np.float64)
    if a.ndim != 2:
        raise ValueError("2-D planes expected")
    h, w = a.shape
    planes = [np.ascontiguousarray(p, dtype=np.float64) for p in (uy, tx, ty)]
    sup = np.ascontiguousarray(support, dtype=np.uint8)
    if any(p.shape != (h, w) for p in planes) or sup.shape != (h, w):
        raise ValueError("planes of different shapes")
    ok = np.empty((h, w), np.uint8)
    n = np.empty((h, w), np.int32)
    eng._call("ofc_local_affine_agreement", w, h, _ptr(a, c_double_p), _ptr(planes[0], c_double_p),
              _ptr(sup, c_u8_p), _ptr(planes[1], c_double_p), _ptr(planes[2], c_double_p), float(radius),
              int(min_support), float(tol), _ptr(ok, c_u8_p), _ptr(n, _abi.c_i32_p))
    return ok.astype(bool), n.astype(np.int64)


def track_pair_device(I1, I2, cfg=None, mask=None, init=None, stream=None, engine=None):
    """track_pair on device-resident torch tensors (float32 images, optional uint8/bool ROI and init fields):
    ofc_track_pair_device on ``stream`` (a torch.cuda.Stream; None = the engine's own stream, synchronised
    before returning). Returns a dict of device tensors named as the pair outputs."""
    import torch
    if I1.shape != I2.shape or I1.dim() != 2:
        raise ValueError(f"image sizes differ or are not 2-D: {tuple(I1.shape)} vs {tuple(I2.shape)}")
    cfg, c = _prep_cfg(cfg)
    h, w = I1.shape
    dev = I1.device
    a = I1.to(torch.float32).contiguous()
    b = I2.to(dev, torch.float32).contiguous()
    m = None if mask is None else mask.to(dev, torch.uint8).contiguous()
    iu = iv = None
    if init is not None:
        iu = init[0].to(dev, torch.float32).contiguous()
        iv = init[1].to(dev, torch.float32).contiguous()
    outs = {k: torch.empty((h, w), dtype=torch.uint8 if k == "valid" else torch.float32, device=dev)
            for k in _abi.PAIR_FIELDS}
    o = OfcPairOut()
    for k, t in outs.items():
        setattr(o, k, ctypes.cast(t.data_ptr(), c_u8_p if k == "valid" else c_float_p))
    eng = engine or default_engine(dev.index or 0)
    p = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())
    eng._call("ofc_track_pair_device", p(a), p(b), w, h, p(m), p(iu), p(iv), ctypes.byref(c), ctypes.byref(o),
              ctypes.c_void_p(stream.cuda_stream) if stream is not None else None)
    if stream is None:
        torch.cuda.synchronize(dev)
    return outs
