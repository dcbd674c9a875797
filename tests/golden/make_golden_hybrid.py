"""Writes tests/golden/hybrid.npz from the reference's own Python hybrid sequence mode
(python/optflow_ref/track.py:331-503):

1. ``_local_affine_agreement`` (track.py:331-382) on seeded planes: a displacement plane with a hole in the support
   (the case of rust/crates/optflow-core/src/track/hybrid.rs:585-633) at several radii, tolerances and supports, and a
   non-square field with a displacement step, noise and a random support at radius 6.5 (rounds to 6, ties to even).
2. ``track_sequence(seq_mode="hybrid")`` on the scripted legs of tests/hybrid_scripts.py, with the reference's
   track_pair replaced the way its tests replace it (python/tests/test_hybrid.py:38-52), ref_update_conf set anew
   before every frame as the scenario lists it.
3. ``track_sequence(seq_mode="hybrid")`` on seeded frames made with the reference's generator (optflow_ref.synth): a
   pattern under a growing uniform strain whose 28 x 30 px patch fades into a second pattern (the direct legs from
   frame 0 lose it, the adjacent legs keep it), an ROI; one run with the reference kept at frame 0, one with
   ref_update_conf 0.9 (the reference moves). Frames are rounded to float32 first (what the C ABI takes).
4. The reference's committed hybrid fixtures (rust/crates/optflow-core/tests/fixtures/hyb_frames.npy, hybA_*.npy,
   hybB_*.npy and meta.json's "hybrid" records, made by its python/bench/make_parity_fixtures.py:436-460 and checked
   by its parity_track.rs:531-638), copied as they are: eight 112 x 112 frames of a translation with a foreign block,
   tracked with ref_update_conf 0.8 and fb_max 10 (A) or 2 (B).

Run in a checkout that has the reference: ``python tests/golden/make_golden_hybrid.py [/path/to/reference]``
(or the OPTFLOW_REFERENCE environment variable).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OPTFLOW_REFERENCE")
if not REF:
    sys.exit("usage: pass the reference checkout as the first argument (or set OPTFLOW_REFERENCE)")
sys.path.insert(0, os.path.join(REF, "python"))
sys.path.insert(0, os.path.dirname(HERE))

import hybrid_scripts as S  # noqa: E402
from optflow_ref import synth  # noqa: E402
from optflow_ref import track as T  # noqa: E402
from optflow_ref.config import Config  # noqa: E402


def f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


def laa_cases(out):
    w = h = 40
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    px, py = 0.5 + 0.01 * xx - 0.02 * yy, -1.0 + 0.015 * yy
    hole = (xx >= 15) & (xx < 25) & (yy >= 15) & (yy < 25)
    sup = ~hole
    ux, uy = np.where(sup, px, np.nan), np.where(sup, py, np.nan)
    cases = [(0.0, 12.0, 20, 0.5), (0.4, 12.0, 20, 0.5), (0.6, 12.0, 20, 0.5), (0.0, 2.0, 20, 0.5),
             (0.0, 8.0, 20, 0.5), (0.0, 8.0, 100000, 0.5), (0.3, 3.5, 5, 0.25)]
    out["laa_plane_ux"], out["laa_plane_uy"], out["laa_plane_support"] = ux, uy, sup.astype(np.uint8)
    out["laa_plane_px"], out["laa_plane_py"] = px, py
    out["laa_plane_cases"] = np.array(cases)
    for c, (dx, radius, ms, tol) in enumerate(cases):
        ok, n = T._local_affine_agreement(ux, uy, sup, px + dx, py, radius, ms, tol)
        out[f"laa_plane_ok{c}"], out[f"laa_plane_n{c}"] = ok.astype(np.uint8), n.astype(np.int32)
    # a displacement step at x = 40 (a crack), noise, a random support; targets off by up to 0.6 px
    rng = np.random.default_rng(8)
    h, w = 64, 80
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    ux = 0.5 + 0.01 * xx - 0.004 * yy + np.where(xx >= 40, 1.5, 0.0) + 0.05 * rng.normal(size=(h, w))
    uy = -0.2 + 0.006 * yy + 0.05 * rng.normal(size=(h, w))
    sup = rng.random((h, w)) < 0.7
    tx, ty = ux + rng.uniform(-0.6, 0.6, (h, w)), uy + rng.uniform(-0.3, 0.3, (h, w))
    ok, n = T._local_affine_agreement(np.where(sup, ux, np.nan), np.where(sup, uy, np.nan), sup, tx, ty, 6.5, 20, 0.5)
    out.update(laa_step_ux=ux, laa_step_uy=uy, laa_step_support=sup.astype(np.uint8), laa_step_tx=tx, laa_step_ty=ty,
               laa_step_ok=ok.astype(np.uint8), laa_step_n=n.astype(np.int32))


def scripted(out):
    name_box = [None]

    def fake(I1, I2, cfg, mask=None, init=None):
        i, j = int(I1[0, 0]), int(I2[0, 0])
        ux, uy, c = S.leg(name_box[0], i, j)
        return T.Result(ux, uy, c, {}, ux, uy, {"coarse": 0.0, "fine": 0.0})

    real = T.track_pair
    T.track_pair = fake
    try:
        for name, (n, _, _, _, _) in S.SCENARIOS.items():
            name_box[0] = name
            cfg = Config(**S.config_keys(name))
            ruc = S.ruc_list(name)
            gen = T.track_sequence(S.frames(n), cfg)
            for k in range(1, n):
                cfg.ref_update_conf = ruc[k - 1]
                kk, r = next(gen)
                assert kk == k
                p = f"s_{name}_{k}_"
                out[p + "fb"] = r.fb.astype(np.int16)
                for q in ("ux", "uy", "conf", "raw_ux", "raw_uy"):
                    out[p + q] = np.float32(getattr(r, q))
                out[p + "timing"] = np.array([r.timing[q] for q in ("reference", "mean_conf", "n_fb_max",
                                                                    "fallback_frac", "fb_gate_rejected",
                                                                    "reacquired")], np.float64)
    finally:
        T.track_pair = real


def real_frames(out):
    n, K = 128, 5
    pat = synth.make_pattern(n, n, seed=21)
    pat2 = synth.make_pattern(n, n, seed=77)
    P = (slice(48, 76), slice(50, 80))
    fr = []
    for j in range(K):
        A = synth.uniform_strain(0.004 * j, -0.002 * j, (n / 2, n / 2), t=(0.7 * j, 0.4 * j))
        a, b = synth.render(pat, n, n, A), synth.render(pat2, n, n, A)
        al = min(1.0, 0.25 * j)
        img = a.copy()
        img[P] = (1 - al) * a[P] + al * b[P]
        fr.append(f32(synth.degrade(img, seed=j, noise=0.005, bits=8)))
    roi = np.zeros((n, n), bool)
    roi[12:-12, 16:-16] = True
    out["r_frames"], out["r_roi"] = np.float32(fr), roi.astype(np.uint8)
    for tag, ruc in (("a", 0.0), ("b", 0.9)):
        t = time.time()
        for k, r in T.track_sequence(fr, Config(seq_mode="hybrid", fb_max=3, ref_update_conf=ruc), mask=roi):
            p = f"r{tag}{k}_"
            out[p + "fb"] = r.fb.astype(np.int16)
            for q in ("ux", "uy", "conf", "raw_ux", "raw_uy"):
                out[p + q] = np.float32(getattr(r, q))
            for q in ("Exx", "Eyy", "Exy", "gmax", "vol"):
                out[p + q] = np.float32(r.strain[q])
            out[p + "timing"] = np.array([r.timing[q] for q in ("reference", "mean_conf", "n_fb_max", "fallback_frac",
                                                                "fb_gate_rejected", "reacquired")], np.float64)
        print(f"real run {tag}: {time.time() - t:.1f} s")


def ref_fixtures(out):
    import json
    fx = os.path.join(REF, "rust", "crates", "optflow-core", "tests", "fixtures")
    load = lambda n: np.load(os.path.join(fx, n + ".npy"))
    out["f_frames"] = np.float32(load("hyb_frames"))
    out["f_A_ux"], out["f_A_conf"], out["f_B_ux"] = (np.float32(load(n)) for n in ("hybA_ux", "hybA_conf", "hybB_ux"))
    out["f_A_fb"], out["f_B_fb"] = (load(n).astype(np.int16) for n in ("hybA_fb", "hybB_fb"))
    with open(os.path.join(fx, "meta.json")) as fh:
        meta = json.load(fh)["hybrid"]
    for name in ("A", "B"):
        out[f"f_{name}_timing"] = np.array([[t[q] for q in ("reference", "mean_conf", "n_fb_max", "fallback_frac",
                                                             "fb_gate_rejected", "reacquired")] for t in meta[name]])


def main():
    out = {}
    laa_cases(out)
    scripted(out)
    real_frames(out)
    ref_fixtures(out)
    np.savez_compressed(os.path.join(HERE, "hybrid.npz"), **out)
    print("hybrid.npz written")


if __name__ == "__main__":
    main()
