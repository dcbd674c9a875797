"""Device timings of the sequence-side components on synthetic inputs (one JSON line per workload).

    PYTHONPATH=optflow-soil_b200 python -m optflow_b200.measure [frames] [tavg] [hybrid] [stream] [pairs] [pipeline] ...

Every workload is rendered on the GPU (optflow_b200.synth, seeded) and timed after one warm-up run: wall times with
host perf_counter around the call, device times with the engine's per-kernel CUDA events (ofc_set_profile /
ofc_profile_read) in a separate run, since the profile mode waits for every replayed graph.

  frames  rgb24 1920 x 1080 frames (the video the CLI reads) through to_gray with scale 2: k_to_gray's device time and
          its algorithmic bytes (3 B in and 4 / scale^2 B out per input pixel) against the copy bandwidth
  tavg    average_window of 7 drifting 960 x 540 frames aligned to the centre with the affine model
  hybrid  a 512^2 hybrid sequence (6 frames, a patch fading into another pattern, the reference moving): the legs'
          share and the hybrid state machine's (k_hyb_*, k_laa_*) of the device time
  stream  the CLI's seq loop on 8 rgb24 1920 x 1080 frames at scale 2 (track_stream, chain): wall time per frame
          against the device time of the frame's kernels
  pairs   24 pairs of sides drawn from {256, ..., 2048} (seed 11): one track_pairs call against one track_pair call each
  pipeline  23 rgb24 1920 x 1080 frames, scale 2, step 5, tavg 3, hybrid: the window means inside the streamed driver
          against iter_frames feeding it
  learned[:n]  n (500) held-out 2048^2 pairs of the learned proposal's distribution: POC + refine against the learned
          proposal + refine (device time, error against the known field, fallback counters)
  footing[:n]  the footing-in-sand clip (n = 600 frames of 1920 x 1080) through the streamed hybrid driver
  batch64  the 64 uneven pairs of batch.batch_specs (seed 11): track_pairs against one track_pair call each
  warp    the warp of a 2048^2 plane: the gather kernel against the TMA-staged one
  accumulate  refine's sums on a 2048^2 pair: the gather accumulate against the TMA-staged one
"""
import ctypes
import json
import os
import sys
import time

import numpy as np

from . import synth
from .api import default_engine, track_pair, track_pairs, track_sequence
from .config import Config
from .stream import to_gray, track_stream
from .tavg import average_window

FALLBACK_HBM_GBS = 6650.0


def hbm_peak():
    """The measured copy bandwidth (MEASURED_PEAKS.json at the repository root) or the fallback."""
    root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    try:
        with open(os.path.join(root, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
        for k in ("hbm_gbs", "hbm_GBs", "copy_gbs"):
            if k in peaks:
                return float(peaks[k]), "measured"
    except (OSError, ValueError):
        pass
    return FALLBACK_HBM_GBS, "fallback"


class Profile:
    """Per-kernel device times of the engine's launches between start() and read()."""

    def __init__(self, eng):
        self.eng = eng

    def start(self):
        self.eng.lib.ofc_set_profile(self.eng.handle, b"")
        self.eng.lib.ofc_profile_read(self.eng.handle, None, 0, None, None, 0)

    def read(self):
        cap = 512
        names = ctypes.create_string_buffer(cap * 96)
        counts = (ctypes.c_uint64 * cap)()
        ms = (ctypes.c_double * cap)()
        n = self.eng.lib.ofc_profile_read(self.eng.handle, names, 96, counts, ms, cap)
        self.eng.lib.ofc_set_profile(self.eng.handle, None)
        out = {}
        for i in range(max(n, 0)):
            nm = names.raw[i * 96:(i + 1) * 96].split(b"\0", 1)[0].decode()
            out[nm] = (int(counts[i]), float(ms[i]))
        return out


def _top(prof, k=6):
    tot = sum(v[1] for v in prof.values()) or 1.0
    return [{"kernel": n, "launches": c, "ms": round(t, 3), "share": round(t / tot, 3)}
            for n, (c, t) in sorted(prof.items(), key=lambda kv: -kv[1][1])[:k]]


def _frames_rgb24(n, h=1080, w=1920, seed=3):
    """n rgb24 frames of a speckle pattern drifting by (0.6, 0.3) px per frame, colour-jittered, 8 bit."""
    p = synth.make_pattern(h, w, seed=seed, rmin=1.5, rmax=2.5)
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        g = synth.render(p, h, w, synth.Field(t=(0.6 * k, 0.3 * k), c=(w / 2, h / 2)))
        rgb = np.clip(np.rint(255 * g[..., None] + rng.normal(0, 2, (h, w, 3))), 0, 255).astype(np.uint8)
        out.append(rgb)
    return out


def frames(eng):
    fr = _frames_rgb24(4)
    to_gray(fr[0], 2, engine=eng)
    prof = Profile(eng)
    prof.start()
    t = time.perf_counter()
    for f in fr:
        to_gray(f, 2, engine=eng)
    wall = (time.perf_counter() - t) / len(fr)
    p = prof.read()
    c, ms = next((v for k, v in p.items() if k.startswith("k_to_gray")), (len(fr), float("nan")))
    per = ms / max(c, 1)
    h, w = fr[0].shape[:2]
    byts = 3 * h * w + 4 * (h // 2) * (w // 2)
    peak, src = hbm_peak()
    gbs = byts / (per * 1e-3) / 1e9
    return {"workload": "frames: rgb24 1920x1080 -> grey 960x540 (to_gray, scale 2)", "kernel_ms": round(per, 4),
            "bytes_per_launch": byts, "achieved_gbs": round(gbs, 1), "peak_gbs": peak, "peak_source": src,
            "frac": round(gbs / peak, 3), "wall_ms_per_frame": round(1e3 * wall, 2),
            "note": "wall time includes the pageable host-to-device copy of the 6.2 MB frame"}


def tavg(eng):
    h, w = 540, 960
    p = synth.make_pattern(h, w, seed=5, rmin=1.5, rmax=2.5)
    fr = [synth.degrade(synth.render(p, h, w, synth.Field(t=(0.5 * k, 0.25 * k), c=(w / 2, h / 2)), engine=eng),
                        seed=k, noise=0.004, bits=8) for k in range(7)]
    cfg = Config(max_disp=8.0)
    average_window(fr, 3, align=True, cfg=cfg, engine=eng)
    prof = Profile(eng)
    prof.start()
    t = time.perf_counter()
    average_window(fr, 3, align=True, cfg=cfg, engine=eng)
    wall = time.perf_counter() - t
    pr = prof.read()
    return {"workload": "tavg: mean of 7 drifting 960x540 frames aligned to the centre (affine)",
            "wall_ms": round(1e3 * wall, 2), "device_ms": round(sum(v[1] for v in pr.values()), 3), "top": _top(pr)}


def hybrid(eng):
    n = 512
    p1 = synth.make_pattern(n, n, seed=21, rmin=1.5, rmax=2.5)
    p2 = synth.make_pattern(n, n, seed=77, rmin=1.5, rmax=2.5)
    P = (slice(190, 300), slice(200, 320))
    fr = []
    for j in range(6):
        f = synth.uniform_strain(0.004 * j, -0.002 * j, (n / 2, n / 2), t=(0.7 * j, 0.4 * j))
        a, b = synth.render(p1, n, n, f, engine=eng), synth.render(p2, n, n, f, engine=eng)
        al = min(1.0, 0.25 * j)
        img = a.copy()
        img[P] = (1 - al) * a[P] + al * b[P]
        fr.append(synth.degrade(img, seed=j, noise=0.005, bits=8))
    roi = np.zeros((n, n), bool)
    roi[40:-40, 48:-48] = True
    cfg = Config(seq_mode="hybrid", fb_max=3, ref_update_conf=0.9)
    list(track_sequence(fr, cfg, mask=roi, engine=eng))
    # wall time without the profile mode (whose per-launch events wait for every replayed graph, which would
    # serialise the adjacent leg that runs beside the direct one), then the kernels' device times
    t = time.perf_counter()
    res = list(track_sequence(fr, cfg, mask=roi, engine=eng))
    wall = time.perf_counter() - t
    prof = Profile(eng)
    prof.start()
    list(track_sequence(fr, cfg, mask=roi, engine=eng))
    pr = prof.read()
    tot = sum(v[1] for v in pr.values())
    hyb = sum(v[1] for k, v in pr.items() if k.startswith("k_hyb") or k.startswith("k_laa"))
    return {"workload": "hybrid: 512^2, 6 frames, fading patch, ref_update_conf 0.9, fb_max 3",
            "wall_ms_per_frame": round(1e3 * wall / (len(fr) - 1), 2), "device_ms_per_frame": round(tot / (len(fr) - 1), 3),
            "hybrid_state_share": round(hyb / tot, 4), "hybrid_state_ms_per_frame": round(hyb / (len(fr) - 1), 3),
            "references": [r.timing["reference"] for _, r in res],
            "fallback_frac": [round(r.timing["fallback_frac"], 4) for _, r in res],
            "top": _top({k: v for k, v in pr.items() if k.startswith("k_hyb") or k.startswith("k_laa")})}


def stream(eng):
    fr = _frames_rgb24(8, seed=9)
    cfg = Config()
    list(track_stream(fr[:3], cfg, scale=2, engine=eng))
    t = time.perf_counter()
    res = list(track_stream(fr, cfg, scale=2, engine=eng))
    wall = time.perf_counter() - t
    prof = Profile(eng)
    prof.start()
    list(track_stream(fr, cfg, scale=2, engine=eng))
    pr = prof.read()
    tot = sum(v[1] for v in pr.values())
    k = len(res)
    return {"workload": "stream: 8 rgb24 1920x1080 frames, scale 2, chain (track_stream)",
            "frames_tracked": k, "wall_ms_per_frame": round(1e3 * wall / k, 2),
            "device_ms_per_frame": round(tot / k, 3),
            "to_gray_ms_per_frame": round(sum(v[1] for n, v in pr.items() if n.startswith("k_to_gray")) / len(fr), 4)}


def pairs(eng):
    n = 2048
    p = synth.make_pattern(n, n, seed=7, rmin=1.5, rmax=2.5)
    a = synth.degrade(synth.render(p, n, n, None, engine=eng), seed=1, noise=0.01, bits=8)
    b = synth.degrade(synth.render(p, n, n, synth.Field(A=((1.01, 0.003), (0.003, 0.996)), c=(n / 2, n / 2), amp=1.5,
                                                          wavelength=256.0, s=(1.0, 1.0)), engine=eng),
                      seed=2, noise=0.01, bits=8)
    rng = np.random.default_rng(11)
    sides = [256, 512, 768, 1024, 1536, 2048]
    items = []
    for _ in range(24):
        h, w = int(rng.choice(sides)), int(rng.choice(sides))
        items.append((a[:h, :w], b[:h, :w]))
    px = sum(it[0].size for it in items)
    cfg = Config()
    track_pairs(items, cfg, engine=eng)
    [track_pair(x, y, cfg, engine=eng) for x, y in items]
    t = time.perf_counter()
    [track_pair(x, y, cfg, engine=eng) for x, y in items]
    t1 = time.perf_counter() - t
    t = time.perf_counter()
    track_pairs(items, cfg, engine=eng)
    t2 = time.perf_counter() - t
    return {"workload": "pairs: 24 crops with sides from {256..2048} (seed 11)", "megapixels": round(px / 1e6, 2),
            "one_call_each_s": round(t1, 3), "one_call_each_mpx_s": round(px / t1 / 1e6, 1),
            "track_pairs_s": round(t2, 3), "track_pairs_mpx_s": round(px / t2 / 1e6, 1)}


def pipeline(eng):
    """The CLI's recommended sequence settings on video frames: rgb24 1920 x 1080, scale 2, step 5, tavg 3, hybrid;
    the window means made inside the streamed driver against iter_frames (grey frames back to the host, each window
    uploaded again) feeding the same driver."""
    from .stream import iter_frames
    fr = _frames_rgb24(23, seed=13)
    cfg = Config(seq_mode="hybrid")
    kw = dict(step=5, tavg=3)
    list(track_stream(fr[:12], cfg, scale=2, engine=eng, **kw))
    t = time.perf_counter()
    a = list(track_stream(fr, cfg, scale=2, engine=eng, **kw))
    t_dev = time.perf_counter() - t
    t = time.perf_counter()
    b = list(track_stream(iter_frames(iter(fr), scale=2, cfg=cfg, engine=eng, **kw), cfg, engine=eng))
    t_host = time.perf_counter() - t
    same = all(np.array_equal(x.ux, y.ux, equal_nan=True) for (_, x), (_, y) in zip(a, b))
    return {"workload": "pipeline: 23 rgb24 1920x1080 frames, scale 2, step 5, tavg 3, hybrid (5 tracked frames)",
            "results": len(a), "wall_ms_per_result_device_windows": round(1e3 * t_dev / len(a), 2),
            "wall_ms_per_result_iter_frames": round(1e3 * t_host / max(len(b), 1), 2), "identical": bool(same)}


def _device_pair_ms(eng, d_a, d_b, n_w, n_h, reps=3, d_roi=None):
    """Device time (CUDA events, median of reps after one untimed run) of one pair through ofc_track_pair_device on
    device-resident inputs, and its outputs (host arrays)."""
    import torch
    from . import _abi
    dev = d_a.device
    outs = {k: torch.empty((n_h, n_w), dtype=torch.uint8 if k == "valid" else torch.float32, device=dev)
            for k in _abi.PAIR_FIELDS}
    po = _abi.OfcPairOut()
    for k, t in outs.items():
        setattr(po, k, ctypes.cast(t.data_ptr(), _abi.c_u8_p if k == "valid" else _abi.c_float_p))
    c = Config().to_ofc()
    stream = torch.cuda.Stream(dev)
    err = ctypes.create_string_buffer(1024)

    def run():
        st = eng.lib.ofc_track_pair_device(eng.handle, d_a.data_ptr(), d_b.data_ptr(), n_w, n_h,
                                           None if d_roi is None else d_roi.data_ptr(), None, None, ctypes.byref(c),
                                           ctypes.byref(po), ctypes.c_void_p(stream.cuda_stream), err, 1024)
        if st != 0:
            raise RuntimeError(err.value.decode())

    run()
    ms = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms.append(e0.elapsed_time(e1))
    return float(np.median(ms)), {k: v.cpu().numpy() for k, v in outs.items()}


def learned(eng, n_pairs=500, size=2048, seed=23):
    """Held-out pairs of the learned proposal's distribution (a Gaussian-process field of length scale 64-512 px
    plus a shear band; optflow_b200.net.random_field) at size^2: plain POC + refine (this engine) against the learned
    proposal + refine (a second engine on the same GPU with the shipped weights), device time per pair (CUDA events,
    inputs resident), RMS error of the valid pixels against the known field, and the proposal's fallback counters."""
    import torch
    from . import net
    from .api import Engine
    rng = np.random.default_rng(seed + 1000003)  # held out: the training set draws from default_rng(seed)
    dev = torch.device("cuda", getattr(eng, "device", 0))
    eng_net = Engine(getattr(eng, "device", 0))
    eng_net.set_coarse_net("default")
    t_poc, t_net, e_poc, e_net, v_poc, v_net = [], [], [], [], [], []
    reps = 3
    for _ in range(n_pairs):
        a, b, field = net.training_pair(rng, size, size, engine=eng)
        tu, tv = field.displacement(size, size)
        d_a, d_b = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
        ms0, o0 = _device_pair_ms(eng, d_a, d_b, size, size, reps)
        ms1, o1 = _device_pair_ms(eng_net, d_a, d_b, size, size, reps)
        t_poc.append(ms0)
        t_net.append(ms1)
        for o, e, v in ((o0, e_poc, v_poc), (o1, e_net, v_net)):
            m = o["valid"].astype(bool)
            du, dv = o["ux"][m] - tu[m], o["uy"][m] - tv[m]
            e.append(float(np.sqrt(np.mean(du * du + dv * dv))) if m.any() else float("nan"))
            v.append(float(m.mean()))
    st = eng_net.coarse_net_stats()
    runs = reps + 1  # every pair runs once untimed and reps times timed, with the same outcome
    fb = {k: int(v) // runs for k, v in st.items()}
    px = size * size
    e_poc, e_net = np.array(e_poc), np.array(e_net)
    return {"workload": f"learned: {n_pairs} held-out {size}^2 pairs (GP field 64-512 px + shear band, seed {seed})",
            "poc_ms_per_pair": round(float(np.mean(t_poc)), 3), "learned_ms_per_pair": round(float(np.mean(t_net)), 3),
            "poc_pixel_pairs_s": px / (np.mean(t_poc) / 1e3), "learned_pixel_pairs_s": px / (np.mean(t_net) / 1e3),
            "poc_rms_px": round(float(np.nanmean(e_poc)), 5), "learned_rms_px": round(float(np.nanmean(e_net)), 5),
            "poc_rms_px_median": round(float(np.nanmedian(e_poc)), 5),
            "learned_rms_px_median": round(float(np.nanmedian(e_net)), 5),
            "pairs_within_0.02px": {"poc": int(np.sum(e_poc <= 0.02)), "learned": int(np.sum(e_net <= 0.02))},
            "valid_fraction": {"poc": round(float(np.mean(v_poc)), 4), "learned": round(float(np.mean(v_net)), 4)},
            "fallback": fb}


def footing(eng, n_frames=600):
    """The footing-in-sand clip (synth.footing_field): 1920 x 1080 uint8 frames (speckle seed 31, noise 0.008),
    rendered first on a second engine (timed apart), then tracked from host memory with the CLI's recommended video settings (scale 2,
    step 5, seq_mode hybrid, tavg 3, prewarp_freeze_at 3) over the sand below the surface; wall time per result, the
    RMS error of the valid pixels against the known field (on the downscaled grid), and the share of ROI pixels carried
    by the adjacent leg."""
    from .api import Engine
    h, w, sc, step, tavg, surface = 1080, 1920, 2, 5, 3, 300.0
    rend = Engine(getattr(eng, "device", 0))
    p = synth.make_pattern(h, w, seed=31, rmin=1.5, rmax=2.5)

    t = time.perf_counter()
    clip = [np.round(synth.degrade(synth.render(p, h, w, synth.footing_field(k, w, h, surface, frames=n_frames),
                                                engine=rend), seed=1000 + k, noise=0.008, bits=8) * 255).astype(np.uint8)
            for k in range(n_frames)]
    t_render = time.perf_counter() - t

    hs, ws = h // sc, w // sc
    roi = np.zeros((hs, ws), bool)
    roi[int(np.ceil(surface / sc)) + 2:, :] = True
    cfg = Config(seq_mode="hybrid", prewarp_freeze_at=3)
    errs, fbs, valid, ks = [], [], [], []
    # the downscaled grid's pixel centres in full-resolution coordinates (box downscale of sc x sc blocks)
    yy, xx = np.mgrid[0:hs, 0:ws].astype(np.float64)
    X, Y = sc * xx + (sc - 1) / 2.0, sc * yy + (sc - 1) / 2.0
    t = time.perf_counter()
    got = [(k, r.ux, r.uy, r.fb) for k, r in track_stream(clip, cfg, mask=roi, scale=sc, step=step, tavg=tavg,
                                                           engine=eng)]
    wall = time.perf_counter() - t
    for k, ux, uy, fb in got:
        raw = k * step
        tu, tv = synth.footing_field(raw, w, h, surface, frames=n_frames).displacement_at(X, Y)
        m = np.isfinite(ux)
        du, dv = ux[m] - tu[m] / sc, uy[m] - tv[m] / sc
        errs.append(float(np.sqrt(np.mean(du * du + dv * dv))) if m.any() else float("nan"))
        valid.append(float(m[roi].mean()))
        fbs.append(float((fb[roi] > 0).mean()) if fb is not None else 0.0)
        ks.append(raw)
    n = len(errs)
    return {"workload": f"footing: {n_frames} 1920x1080 uint8 frames, scale 2, step 5, hybrid, tavg 3, "
                        f"prewarp_freeze_at 3, sand ROI ({n} results)",
            "results": n, "wall_ms_per_result": round(1e3 * wall / max(n, 1), 2),
            "render_s_all_frames": round(t_render, 1),
            "rms_px_downscaled": {"mean": round(float(np.nanmean(errs)), 4), "max": round(float(np.nanmax(errs)), 4),
                                  "last": round(errs[-1], 4)},
            "valid_share_of_roi": {"mean": round(float(np.mean(valid)), 4), "min": round(float(np.min(valid)), 4)},
            "adjacent_leg_share": {"mean": round(float(np.mean(fbs)), 4), "max": round(float(np.max(fbs)), 4)},
            "settlement_px_last": round(0.05 * ks[-1], 2)}


def batch64(eng, n=64):
    """The uneven batch of independent pairs (batch.batch_specs: 64 pairs from seed 11, sides drawn from
    {256, ..., 2048}, random affine strain |e| <= 0.02, translation <= 6 px, noise 0.003-0.02): one track_pairs call
    (worker lanes with their own streams and graphs, the FFT plan table installed) against one track_pair call each,
    wall time with the pairs on the host; every result equal between the two."""
    from .batch import batch_specs, make_pair
    specs = batch_specs(n, 11)
    items = [make_pair(s, engine=eng)[:2] for s in specs]
    px = sum(s.pixels for s in specs)
    cfg = Config()
    r_batch = track_pairs(items, cfg, engine=eng)  # warm-up: buffers, plans and graphs
    r_one = [track_pair(x, y, cfg, engine=eng) for x, y in items]
    t = time.perf_counter()
    [track_pair(x, y, cfg, engine=eng) for x, y in items]
    t1 = time.perf_counter() - t
    t = time.perf_counter()
    r_batch = track_pairs(items, cfg, engine=eng)
    t2 = time.perf_counter() - t
    same = all(np.array_equal(a.ux, b.ux, equal_nan=True) for a, b in zip(r_batch, r_one))
    return {"workload": f"batch64: {n} pairs of uneven sides from {{256..2048}} (seed 11)",
            "megapixels": round(px / 1e6, 2), "one_call_each_s": round(t1, 3),
            "one_call_each_pixel_pairs_s": px / t1, "track_pairs_s": round(t2, 3), "track_pairs_pixel_pairs_s": px / t2,
            "identical": bool(same)}


def _smooth_field(n, amp, seed=1):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    ph = rng.uniform(0, 2 * np.pi, 2)
    return (amp * np.sin(xx / 137.0 + ph[0]) * np.cos(yy / 153.0),
            amp * np.cos(xx / 129.0 + yy / 161.0 + ph[1]))


def _kernel_ms(eng, run, reps):
    """Per-launch device time of every kernel `run` launches, over `reps` calls after one warm-up call."""
    run()
    prof = Profile(eng)
    prof.start()
    for _ in range(reps):
        run()
    return {k: round(t / c, 4) for k, (c, t) in prof.read().items() if c}


def warp(eng, reps=20):
    """The warp of a 2048^2 coefficient plane by a smooth 5 px field: the gather kernel (k_warp, the engine's) against
    the TMA-staged one (k_warp_tma); per-launch device ms and whether the outputs are equal."""
    from . import testing
    n = 2048
    c2 = np.random.default_rng(1).normal(size=(n, n)).astype(np.float32)
    sx, sy = _smooth_field(n, 5.0)
    out = {"workload": "warp: 2048^2 plane, smooth 5 px field", "ms_per_launch": {}}
    res = {}
    for mode in (0, 1):
        res[mode] = testing.warp(c2, sx, sy, mode=mode, engine=eng)
        ms = _kernel_ms(eng, lambda: testing.warp(c2, sx, sy, mode=mode, engine=eng), reps)
        out["ms_per_launch"].update({k: v for k, v in ms.items() if k.startswith("k_warp")})
    out["identical"] = bool(np.array_equal(res[0][0].view(np.uint32), res[1][0].view(np.uint32)))
    out["timeouts"] = res[1][1]
    return out


def accumulate(eng, reps=5):
    """refine's first inner-iteration sums of a 2048^2 speckle pair from a smooth 5 px start field: the gather
    accumulate (k_accumulate, the engine's) against the TMA-staged one (k_accumulate_tma); per-launch device ms, the
    achieved algorithmic bandwidth and whether the sums are equal."""
    from . import testing
    n = 2048
    pat = synth.make_pattern(n, n, seed=7)
    a = synth.render(pat, n, n, None, engine=eng).astype(np.float32)
    b = synth.render(pat, n, n, synth.Field(t=(0.7, -0.4), c=(n / 2, n / 2)), engine=eng).astype(np.float32)
    ux, uy = _smooth_field(n, 5.0)
    cfg = Config()
    F = cfg.n_filters()
    byts = n * n * (16 * F + 104) + (n + 64) ** 2 * 8 * F
    out = {"workload": "accumulate: 2048^2 pair, smooth 5 px start field", "ms_per_launch": {}, "GB_s": {}}
    res = {}
    for mode in (0, 1):
        res[mode] = testing.accumulate(a, b, ux, uy, mode=mode, cfg=cfg, engine=eng)
        ms = _kernel_ms(eng, lambda: testing.accumulate(a, b, ux, uy, mode=mode, cfg=cfg, engine=eng), reps)
        for k, v in ms.items():
            if k.startswith("k_accumulate"):
                out["ms_per_launch"][k] = v
                out["GB_s"][k] = round(byts / (v * 1e-3) / 1e9, 1)
    out["identical"] = bool(np.array_equal(res[0][0], res[1][0], equal_nan=True))
    out["timeouts"] = res[1][1]
    return out


WORKLOADS = {"frames": frames, "tavg": tavg, "hybrid": hybrid, "stream": stream, "pairs": pairs, "pipeline": pipeline,
             "learned": learned, "footing": footing, "batch64": batch64, "warp": warp, "accumulate": accumulate}


def main(argv=None):
    """Workload names, optionally with a count (learned:64 runs 64 held-out pairs, footing:100 the first 100
    frames); no name: every workload but learned and footing."""
    names = (argv if argv is not None else sys.argv[1:]) or [k for k in WORKLOADS if k not in ("learned", "footing")]
    eng = default_engine()
    for n in names:
        name, _, cnt = n.partition(":")
        print(json.dumps(WORKLOADS[name](eng, int(cnt)) if cnt else WORKLOADS[name](eng)), flush=True)


if __name__ == "__main__":
    main()
