"""Device timings of the sequence-side components on synthetic inputs (one JSON line per workload).

    PYTHONPATH=optflow-soil_b200 python -m optflow_b200.measure [frames] [tavg] [hybrid] [stream] [pairs] [pipeline]

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


WORKLOADS = {"frames": frames, "tavg": tavg, "hybrid": hybrid, "stream": stream, "pairs": pairs, "pipeline": pipeline}


def main(argv=None):
    names = (argv if argv is not None else sys.argv[1:]) or list(WORKLOADS)
    eng = default_engine()
    for n in names:
        print(json.dumps(WORKLOADS[n](eng)), flush=True)


if __name__ == "__main__":
    main()
