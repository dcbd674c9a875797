"""Dense local-phase flow + strain throughput (pixel-pairs/s) on a 2048^2 speckle pair.

Workload (one step = one tracked pair: coarse POC pyramid -> dense start -> fine stage (8 outer x 2 inner
iterations, 12 Gabor filters) -> confidence -> guard + strain; default configuration):
  * 2048 x 2048 uint8-quantised speckle pair: blobs of make_pattern(2048, 2048, seed=7, rmin=1.5, rmax=2.5) (mean
    speckle diameter about 4 px), rendered with 4 x 4 supersampling by the reference generator's arithmetic (the
    frames equal the reference's synth.render/degrade output bit for bit: tests/test_gpu_config2.py);
  * deformation x = c + A (X - c) + 1.5 sin(2 pi X / 256) (1, 1), A = [[1.01, 0.003], [0.003, 0.996]] about the
    centre (exx 0.01, eyy -0.004, gxy 0.006), Gaussian noise 0.01, 8-bit quantisation;
  * polygon ROI covering the central 80 % ([204.8, 1843.2]^2).
value: pixel-pairs/s with the inputs resident in device memory (ofc_track_pair_device), device time from CUDA
events around each step, L2 flushed (256 MiB write) between steps; e2e: the same through the host C ABI
(ofc_track_pair) with pinned host buffers, uploads and downloads of the nine CLI outputs included.
--impl reference: the reference's CPU path (the float64 C++/OpenMP oracle, a restatement of it: the Rust CLI cannot
be built here) on all host cores, over the same pair; a step is one window of the reference CLI's own 2 x 2 tiling
of the pair (tile.rs:56,85: 1024 px tiles with a 64 px margin, windows of 1088^2), the four windows in turn, and
the value is the tiles' core pixels per second. That process renders its inputs with the oracle's restatement of
the generator and loads no part of the CUDA engine.

Multi-GPU (torchrun): one independent replica per GPU (the pair path has no exchange step); value = all ranks'
pixels / the slowest rank's time.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "optflow-soil_b200"))

N_PIX = 2048
METRIC = "pixel-pairs/s dense flow+strain at 2048^2 (POC coarse + local-phase refine + guard + strain)"
UNIT = "pixel-pairs/s"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


PAIR_FIELD = dict(A=((1.01, 0.003), (0.003, 0.996)), amp=1.5, wavelength=256.0, s=(1.0, 1.0))


def make_pair(n=N_PIX, engine=None, renderer=None):
    """The benchmark pair: (a, b, roi, field). renderer(pattern, h, w, field) -> float64 image; None: the engine's
    GPU renderer (ofc_synth_render)."""
    from optflow_b200 import synth
    p = synth.make_pattern(n, n, seed=7, rmin=1.5, rmax=2.5)
    c = n / 2.0
    field = synth.Field(c=(c, c), **PAIR_FIELD)
    render = renderer or (lambda pat, h, w, f: synth.render(pat, h, w, f, engine=engine))
    a = synth.degrade(render(p, n, n, None), seed=1, noise=0.01, bits=8)
    b = synth.degrade(render(p, n, n, field), seed=2, noise=0.01, bits=8)
    lo, hi = 0.1 * n, 0.9 * n
    roi = synth.rect_roi(n, n, lo, lo, hi, hi)
    return a, b, roi, field


def workload_config(n):
    """The config object both arms print."""
    return {"workload": f"{n}^2 speckle pair (seed 7, 4 px speckles), affine exx 0.01 eyy -0.004 gxy 0.006 + 1.5 px "
                        f"sinusoid (256 px), noise 0.01, 8 bit, ROI 80 %",
            "steps_are": "one tracked pair each", "l2": "flushed (256 MiB write) between steps"}


class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def hbm_peak():
    try:
        with open(PEAKS) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


# algorithmic bytes of one k_accumulate launch: per pixel the reference pack (float4 per filter), the field
# (ux, uy, sx, sy: float64), its spline (csx, csy), the seven sums written (float64); per padded pixel the
# twelve response planes (complex float32), each read once
def accumulate_bytes(W, H, F=12):
    N, Np = W * H, (W + 64) * (H + 64)
    return N * (16 * F + 32 + 16 + 56) + Np * 8 * F


# DRAM traffic of one k_accumulate launch over its algorithmic bytes, from one ncu capture on the 2048^2 pair
# (dram__bytes_read.sum + dram__bytes_write.sum = 1415.0 + 231.8 MB against 1669.7 MB algorithmic,
# profiles/k_accumulate_2048.txt); at another size the traffic is this ratio times its algorithmic bytes (both
# grow with the pixel and padded-pixel counts)
ACC_TRAFFIC_RATIO = 1646.8 / 1669.7


def tile_windows(n, tile=1024, margin=64):
    """The reference CLI's tiling of an n x n image (rust/crates/optflow-core/src/tile.rs:56,85): (window slices,
    core pixels) per tile, row-major."""
    out = []
    for y0 in range(0, n, tile):
        for x0 in range(0, n, tile):
            y1, x1 = min(y0 + tile, n), min(x0 + tile, n)
            win = (slice(max(y0 - margin, 0), min(y1 + margin, n)), slice(max(x0 - margin, 0), min(x1 + margin, n)))
            out.append((win, (y1 - y0) * (x1 - x0)))
    return out


def run_cpu(a, b, roi, steps, warmup):
    """The oracle on all host threads, one tile window of the pair per step (the four in turn)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from optflow_b200 import Config
    threads = oracle.threads(0)
    wins = tile_windows(a.shape[0])
    px, sec = 0, 0.0
    for i in range(warmup + steps):
        win, core = wins[i % len(wins)]
        t = time.perf_counter()
        oracle.track_pair(a[win], b[win], Config(), mask=roi[win])
        dt = time.perf_counter() - t
        if i >= warmup:
            px += core
            sec += dt
    (wy, wx), core = wins[0][0], wins[0][1]
    return {"value": px / sec, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} step(s), each one of the {len(wins)} windows of the reference CLI's tiling of the "
                      f"{a.shape[0]}^2 pair ({wy.stop - wy.start}x{wx.stop - wx.start}, its {core} core pixels "
                      f"credited), float64 oracle (C++/OpenMP restatement of the reference's pair path), {threads} "
                      f"threads, {sec / steps:.2f} s per window"}


def learned_leg(eng, d_a, d_b, roi, field, n, steps, flush, stream):
    """The pair through the learned coarse proposal (device time per pair, CUDA events, L2 flushed between steps)
    next to the POC path on the same pair: pixel-pairs/s of each, the RMS error of each path's valid pixels against
    the known field, and the proposal's fallback counters."""
    import torch
    from optflow_b200 import Config, Engine, _abi
    dev = d_a.device
    en = Engine(dev.index or 0)
    en.set_coarse_net("default")
    c = Config().to_ofc()
    d_roi = torch.from_numpy(roi.astype(np.uint8)).to(dev)
    tu, tv = field.displacement(n, n)
    res = {}
    for name, e in (("poc", eng), ("learned", en)):
        outs = {k: torch.empty((n, n), dtype=torch.uint8 if k == "valid" else torch.float32, device=dev)
                for k in _abi.PAIR_FIELDS}
        po = _abi.OfcPairOut()
        for k, t in outs.items():
            setattr(po, k, ctypes.cast(t.data_ptr(), _abi.c_u8_p if k == "valid" else _abi.c_float_p))
        err = ctypes.create_string_buffer(1024)

        def step():
            st = e.lib.ofc_track_pair_device(e.handle, d_a.data_ptr(), d_b.data_ptr(), n, n, d_roi.data_ptr(), None,
                                             None, ctypes.byref(c), ctypes.byref(po),
                                             ctypes.c_void_p(stream.cuda_stream), err, 1024)
            if st != 0:
                raise RuntimeError(err.value.decode())

        for _ in range(2):
            step()
        ms = []
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ms.append(e0.elapsed_time(e1))
        m = outs["valid"].cpu().numpy().astype(bool)
        du = outs["ux"].cpu().numpy()[m] - tu[m]
        dv = outs["uy"].cpu().numpy()[m] - tv[m]
        res[name] = {"value": n * n / (float(np.mean(ms)) / 1e3), "unit": UNIT, "ms_per_step": float(np.mean(ms)),
                     "truth_rms_px": float(np.sqrt(np.mean(du * du + dv * dv))), "valid_fraction": float(m.mean())}
    res["learned"]["fallback"] = en.coarse_net_stats()
    en.close()
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--size", type=int, default=N_PIX)
    ap.add_argument("--profile-all", action="store_true", help="print every kernel's device time to stderr")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-proposal leg")
    args = ap.parse_args()
    assert args.warmup >= 0 and args.steps >= 1

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        a, b, roi, _ = make_pair(args.size, renderer=oracle.render)
        base = run_cpu(a, b, roi, args.steps, args.warmup)
        line = {"metric": METRIC, "value": base["value"], "unit": UNIT, "impl": "reference", "n_gpus": 0,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "vs_baseline": None,
                "dtype": "f64", "data": "synthetic", "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "config": workload_config(args.size)}
        print(json.dumps(line), flush=True)
        return

    import torch
    import torch.distributed as dist
    from optflow_b200 import Config, Engine, _abi
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    eng = Engine(local)
    lib = eng.lib
    n = args.size
    a, b, roi, field = make_pair(n, engine=eng)
    cfg = Config()
    c = cfg.to_ofc()

    # device-resident inputs and outputs
    d_a = torch.from_numpy(a).to(dev)
    d_b = torch.from_numpy(b).to(dev)
    d_roi = torch.from_numpy(roi.astype(np.uint8)).to(dev)
    outs = {k: torch.empty((n, n), dtype=torch.uint8 if k == "valid" else torch.float32, device=dev)
            for k in _abi.PAIR_FIELDS}
    dout = _abi.OfcPairOut()
    for k, t in outs.items():
        setattr(dout, k, ctypes.cast(t.data_ptr(), _abi.c_u8_p if k == "valid" else _abi.c_float_p))
    # a stream of its own: the engine reads a null stream handle as "the engine's stream", and torch's
    # legacy default stream has the null handle
    stream = torch.cuda.Stream(dev)
    err = ctypes.create_string_buffer(1024)

    def step():
        st = lib.ofc_track_pair_device(eng.handle, d_a.data_ptr(), d_b.data_ptr(), n, n, d_roi.data_ptr(), None, None,
                                       ctypes.byref(c), ctypes.byref(dout), ctypes.c_void_p(stream.cuda_stream),
                                       err, 1024)
        if st != 0:
            raise RuntimeError(err.value.decode())

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2
    # the profile filter is part of the captured pair graphs' key: set it before the warm-up, which then
    # captures the graphs the timed steps replay
    lib.ofc_set_profile(eng.handle, b"" if args.profile_all else b"k_accumulate")
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    lib.ofc_profile_read(eng.handle, None, 0, None, None, 0)  # clear
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    launches0 = eng.kernel_launches()
    ms = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms.append(e0.elapsed_time(e1))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    launches = eng.kernel_launches() - launches0
    clk = clocks.stop()
    # per-kernel device times of the timed steps (events on the launching stream)
    cap = 256
    names = ctypes.create_string_buffer(cap * 96)
    counts = (ctypes.c_uint64 * cap)()
    kms = (ctypes.c_double * cap)()
    nk = lib.ofc_profile_read(eng.handle, names, 96, counts, kms, cap)
    lib.ofc_set_profile(eng.handle, None)
    prof = {}
    for i in range(max(nk, 0)):
        nm = names.raw[i * 96:(i + 1) * 96].split(b"\0", 1)[0].decode()
        prof[nm] = (int(counts[i]), float(kms[i]))
    if args.profile_all and rank == 0:
        tot = sum(v[1] for v in prof.values())
        for nm, (cnt, t) in sorted(prof.items(), key=lambda kv: -kv[1][1]):
            print(f"{nm:45s} {cnt:6d} launches {t / args.steps:9.3f} ms/step {100 * t / tot:5.1f} %", file=sys.stderr)

    t_step = float(np.mean(ms)) / 1e3
    t_max = t_step
    if world > 1:
        tt = torch.tensor([t_step], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    value = world * n * n / t_max

    # e2e through the host C ABI with pinned buffers (the nine CLI outputs downloaded)
    pin = lambda arr: torch.from_numpy(arr).pin_memory()
    h_a, h_b, h_roi = pin(a), pin(b), pin(roi.astype(np.uint8))
    hout = {k: torch.empty((n, n), dtype=torch.uint8 if k == "valid" else torch.float32).pin_memory()
            for k in ("ux", "uy", "conf", "exx", "eyy", "exy", "gmax", "vol", "valid")}
    hpo = _abi.OfcPairOut()
    for k, t in hout.items():
        setattr(hpo, k, ctypes.cast(t.data_ptr(), _abi.c_u8_p if k == "valid" else _abi.c_float_p))
    h2d = sum(t.numel() * t.element_size() for t in (h_a, h_b, h_roi))
    d2h = sum(t.numel() * t.element_size() for t in hout.values())
    fp = ctypes.POINTER(ctypes.c_float)

    def e2e_step():
        st = lib.ofc_track_pair(eng.handle, ctypes.cast(h_a.data_ptr(), fp), ctypes.cast(h_b.data_ptr(), fp), n, n,
                                ctypes.cast(h_roi.data_ptr(), _abi.c_u8_p), None, None, ctypes.byref(c),
                                ctypes.byref(hpo), err, 1024)
        if st != 0:
            raise RuntimeError(err.value.decode())

    e2e_step()
    if world > 1:
        dist.barrier()
    e2e_t = []
    for _ in range(args.steps):
        t = time.perf_counter()
        e2e_step()
        e2e_t.append(time.perf_counter() - t)
    e2e_sec = float(np.mean(e2e_t))
    if world > 1:
        tt = torch.tensor([e2e_sec], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_sec = float(tt.item())
    valid_frac = float(hout["valid"].numpy().mean())

    # the same pair with the learned coarse proposal in place of POC (a second engine with the shipped weights):
    # device time per pair and the error of both paths against the known field
    learned = None
    if not args.no_learned and os.path.exists(os.path.join(ROOT, "optflow-soil_b200", "optflow_b200", "weights",
                                                           "coarse_net.npz")):
        learned = learned_leg(eng, d_a, d_b, roi, field, n, args.steps, flush, stream)

    line = None
    if rank == 0:
        peak, peak_kind = hbm_peak()
        # the dominant kernel: the TMA-staged accumulate (the gather form where the planes have no tensor maps)
        acc_name = next((k for k in ("k_accumulate_tma", "k_accumulate") if prof.get(k, (0, 0))[0]), None)
        acc = prof.get(acc_name) if acc_name else None
        roof = None
        if acc and acc[0]:
            per_launch_s = acc[1] / acc[0] / 1e3
            byts = accumulate_bytes(n, n, cfg.n_filters())
            achieved = byts / per_launch_s / 1e9
            roof = {"bound": "hbm", "kernel": acc_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_source": peak_kind,
                    "traffic": ACC_TRAFFIC_RATIO * byts,
                    "traffic_source": "ncu capture of this kernel on the 2048^2 pair (ratio to algorithmic bytes)",
                    "algorithmic_bytes_per_launch": byts, "launch_ms": per_launch_s * 1e3,
                    "launches_per_step": acc[0] / args.steps}
        base = None
        if world == 1 and not args.no_cpu:
            base = run_cpu(a, b, roi, 1, 0)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_max * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "fp32 transforms + fp64 sums/solve", "data": "synthetic",
                "config": dict(workload_config(n), parallelism=f"replicas x{world}"), "valid_fraction": valid_frac,
                "e2e": {"value": world * n * n / e2e_sec, "unit": UNIT, "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": e2e_sec * 1e3},
                "gpu_launches": int(launches), "clocks": clk, "roofline": roof, "cpu_baseline": base,
                "learned_vs_poc": learned}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
