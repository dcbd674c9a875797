"""Writes the golden vectors of tests/golden/*.npz by running the reference's own Python specification.

Run in a checkout that has the reference (``python tests/golden/make_golden.py [/path/to/reference]``; the
or the OPTFLOW_REFERENCE environment variable). The reference's ``python/optflow_ref`` package is imported and called on
seeded synthetic inputs made with its own generator (``optflow_ref.synth``); inputs are rounded to float32
first (what the C ABI takes, ``Image<f32>`` in the reference's Rust engine interface) and the reference is
run on exactly those values, so inputs and expected outputs match bit for bit. Outputs are stored as float32
(the precision of the reference CLI's .npy outputs), which is far below every parity tolerance.

The GPU box that runs the parity tests has no copy of the reference, so these files are committed.
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

from optflow_ref import interp, phaseflow, poc, strain, synth, track  # noqa: E402
from optflow_ref.config import Config  # noqa: E402
from scipy.ndimage import distance_transform_edt  # noqa: E402


def f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


def save(name, **arrays):
    out = {}
    for k, v in arrays.items():
        v = np.asarray(v)
        if v.dtype == np.float64:
            v = v.astype(np.float32)
        if v.dtype == np.bool_:
            v = v.astype(np.uint8)
        out[k] = v
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: {sorted(out)}")


class AffineSine:
    """x = c + A (X - c) + t + amp * sin(2 pi X_x / wavelength) * (1, 1): the deformation of the 2048^2
    benchmark pair, here at a smaller size. fwd/inv/grad like the field classes of optflow_ref.synth; inv by
    Newton iteration on the 2 x 2 Jacobian."""

    def __init__(self, A, c, t=(0.0, 0.0), amp=0.0, wavelength=256.0):
        self.aff = synth.Affine(A, t, c)
        self.amp, self.k = amp, 2 * np.pi / wavelength

    def fwd(self, X, Y):
        x, y = self.aff.fwd(X, Y)
        s = self.amp * np.sin(self.k * X)
        return x + s, y + s

    def inv(self, x, y):
        X, Y = self.aff.inv(x, y)
        A = self.aff.A
        for _ in range(30):
            fx, fy = self.fwd(X, Y)
            rx, ry = fx - x, fy - y
            ds = self.amp * self.k * np.cos(self.k * X)
            j00, j01, j10, j11 = A[0, 0] + ds, A[0, 1], A[1, 0] + ds, A[1, 1]
            det = j00 * j11 - j01 * j10
            X = X - (j11 * rx - j01 * ry) / det
            Y = Y - (-j10 * rx + j00 * ry) / det
        return X, Y


def pair_case(name, n, seed, field, noise, roi=None, cfg=None, init=None, foreign=None):
    p = synth.make_pattern(n, n, seed=seed)
    a = synth.render(p, n, n)
    b = synth.render(p, n, n, field)
    if foreign is not None:
        other = synth.render(synth.make_pattern(n, n, seed=77), n, n)
        b[:, foreign[0]:foreign[1]] = other[:, foreign[0]:foreign[1]]
    if noise:
        a = synth.degrade(a, seed=2 * seed + 1, noise=noise, bits=8)
        b = synth.degrade(b, seed=2 * seed + 2, noise=noise, bits=8)
    a, b = f32(a), f32(b)
    cfg = cfg or Config()
    t = time.time()
    r = track.track_pair(a, b, cfg, mask=roi, init=init)
    gx, gy = synth.displacement(field, n, n)
    kw = dict(a=a, b=b, ux=r.ux, uy=r.uy, conf=r.conf, raw_ux=r.raw_ux, raw_uy=r.raw_uy, gt_ux=gx, gt_uy=gy,
              **{k: r.strain[k] for k in ("Exx", "Eyy", "Exy", "gmax", "vol")})
    if roi is not None:
        kw["roi"] = roi
    if init is not None:
        kw["init_ux"], kw["init_uy"] = init
    save(name, **kw)
    print(f"  {time.time() - t:.1f} s, valid {np.isfinite(r.ux).mean():.3f}")


def main():
    rng = np.random.default_rng(2024)

    # interp: B-spline coefficients, samples (incl. clamped coordinates), warp, blur
    img = rng.normal(size=(40, 50))
    x = rng.uniform(-3, 53, 500)
    y = rng.uniform(-3, 43, 500)
    ux, uy = rng.uniform(-2, 2, img.shape), rng.uniform(-2, 2, img.shape)
    save("interp", img=img, x=x.astype(np.float32), y=y.astype(np.float32),
         coeffs=interp.bspline_coeffs(img),
         sample=interp.sample(interp.bspline_coeffs(img), f32(x), f32(y)),
         warp_ux=ux, warp_uy=uy, warp=interp.warp(f32(img), f32(ux), f32(uy)),
         blur4=interp.gauss_blur(f32(img), 4.0), blur1=interp.gauss_blur(f32(img), 1.0))

    # Gabor responses of a 64^2 speckle image (default bank)
    n = 64
    g = f32(synth.render(synth.make_pattern(n, n, seed=3), n, n))
    cfg = Config()
    bank, fx, fy = phaseflow.gabor_bank((n + 64, n + 64), cfg.lam, cfg.scales, cfg.n_orient, cfg.bandwidth,
                                        cfg.dc_cut)
    ref = phaseflow.reference_phase(g, bank, fx, fy)
    save("gabor", img=g, r_re=np.stack([r.real for r, _, _, _ in ref]), r_im=np.stack([r.imag for r, _, _, _ in ref]),
         gx=np.stack([q for _, q, _, _ in ref]), gy=np.stack([q for _, _, q, _ in ref]),
         amp=np.stack([q for _, _, _, q in ref]))

    # EDT distances and feature transform (scipy's tie rule), rising source density
    src = np.stack([rng.uniform(size=(41, 57)) < p for p in (0.003, 0.02, 0.08, 0.3)])
    src[:, 5, 7] = True
    dist = np.stack([distance_transform_edt(~s) for s in src])
    idx = []
    for s in src:
        _, (iy, ix) = distance_transform_edt(~s, return_indices=True)
        idx.append(iy * s.shape[1] + ix)
    save("edt", src=src, dist=dist, idx=np.stack(idx).astype(np.int32))

    # strain: smooth field with NaN holes, displacement gradient and strain fields
    yy, xx = np.mgrid[0:72, 0:90].astype(float)
    sux = 0.012 * xx - 0.004 * yy + 2e-4 * xx * yy + 0.25 * np.sin(xx / 8.0) + 1e-4 * yy ** 2
    suy = 0.005 * xx + 0.008 * yy + 0.15 * np.cos(yy / 6.0) - 1e-4 * xx ** 2
    sux[30:37, 40:52] = np.nan
    suy[30:37, 40:52] = np.nan
    sux[5:9, 70:74] = np.nan
    sux, suy = f32(sux), f32(suy)
    grads = strain.displacement_gradient(sux, suy, 15)
    sf = strain.strain_fields(*grads)
    save("strain", ux=sux, uy=suy, dudx=grads[0], dudy=grads[1], dvdx=grads[2], dvdy=grads[3],
         **{k: sf[k] for k in ("Exx", "Eyy", "Exy", "gmax", "vol")})

    # POC: coarse_flow with one pyramid level (shift beyond a quarter window), with and without a dense guess
    h, w = 192, 256
    p = synth.make_pattern(h, w, seed=5)
    fld = synth.uniform_strain(0.01, -0.006, (w / 2, h / 2), t=(19.3, -7.6))
    a = f32(synth.degrade(synth.render(p, h, w), seed=1, noise=0.005, bits=8))
    b = f32(synth.degrade(synth.render(p, h, w, fld), seed=2, noise=0.005, bits=8))
    gr = poc.coarse_flow(a, b, Config())
    yy, xx = np.mgrid[0:h, 0:w].astype(float)
    gu, gv = f32(17.0 + 0.01 * xx), f32(-6.0 - 0.005 * yy)
    gi = poc.coarse_flow(a, b, Config(), init_dense=(gu, gv))
    sa, sb = a[:, :], f32(np.full((h, w), 0.5))
    gf = poc.coarse_flow(a, sb, Config(), init_dense=(gu, gv))
    dx, dy, pk = poc.poc_shift(a[40:104, 50:114], b[40:104, 70:134])
    save("poc", a=a, b=b, xs=gr.xs, ys=gr.ys, ux=gr.ux, uy=gr.uy, peak=gr.peak,
         init_ux=gu, init_uy=gv, iux=gi.ux, iuy=gi.uy, ipeak=gi.peak, fux=gf.ux, fuy=gf.uy, fpeak=gf.peak,
         shift=np.array([dx, dy, pk]), n_levels=np.array([poc.n_levels(32.0, 64, (h, w))]))

    # refine from a near-exact start, shape orders 1 and 2
    n = 128
    p = synth.make_pattern(n, n, seed=7)
    fld = synth.uniform_strain(0.02, -0.01, (64, 64), t=(1.3, -0.8))
    a, b = f32(synth.render(p, n, n)), f32(synth.render(p, n, n, fld))
    gx, gy = synth.displacement(fld, n, n)
    iu, iv = f32(gx + 0.3), f32(gy - 0.3)
    kw = dict(a=a, b=b, init_ux=iu, init_uy=iv, gt_ux=gx, gt_uy=gy)
    for order in (1, 2):
        fl = phaseflow.refine(a, b, iu, iv, Config(shape_order=order))
        kw.update({f"o{order}_ux": fl.ux, f"o{order}_uy": fl.uy, f"o{order}_conf": fl.conf,
                   f"o{order}_resid": fl.resid})
    save("refine", **kw)

    # refine on a stripe texture: aperture-degenerate, keeps its start, confidence below conf_min
    xs_ = np.arange(64)[None, :] * np.ones((64, 1))
    sa, sb = f32(0.5 + 0.2 * np.sin(xs_ / 2)), f32(0.5 + 0.2 * np.sin((xs_ - 1.0) / 2))
    iu, iv = np.full(sa.shape, 0.7), np.full(sa.shape, -0.4)
    fl = phaseflow.refine(sa, sb, iu, iv, Config())
    save("stripe", a=sa, b=sb, init_ux=iu, init_uy=iv, ux=fl.ux, uy=fl.uy, conf=fl.conf)

    # refine with the edge guard off: only matches that leave image 2 get confidence 0
    n = 64
    p = synth.make_pattern(n, n, seed=13)
    fld = synth.uniform_strain(0.004, -0.002, (32.0, 32.0), t=(-1.5, 1.7))
    a, b = f32(synth.render(p, n, n)), f32(synth.render(p, n, n, fld))
    gx, gy = synth.displacement(fld, n, n)
    iu, iv = f32(gx + 0.3), f32(gy - 0.3)
    fl = phaseflow.refine(a, b, iu, iv, Config(edge_guard=0.0))
    save("border", a=a, b=b, init_ux=iu, init_uy=iv, ux=fl.ux, uy=fl.uy, conf=fl.conf)

    # track_pair: translation + strain, a foreign band (a large low-confidence source) and a rectangular ROI
    n = 160
    roi = np.zeros((n, n), bool)
    roi[12:150, 8:152] = True
    pair_case("pair_roi", n, 21, synth.uniform_strain(0.01, -0.005, (80, 80), t=(5.1, -2.2)), 0.005, roi=roi,
              foreign=(72, 88))

    # the 256^2 case of the CPU-runnable workload: frame 0 -> frame 2 of the strain sequence
    # (make_pattern(256, 256, seed=1); uniform strain 0.005 k about (128, 128) plus (0.8 k, 0) px; noise 0.005)
    n, k = 256, 2
    p = synth.make_pattern(n, n, seed=1)
    fr = [synth.degrade(synth.render(p, n, n, synth.uniform_strain(0.005 * j, 0.0, (128, 128), t=(0.8 * j, 0.0))),
                        seed=j, noise=0.005, bits=8) for j in (0, k)]
    a, b = f32(fr[0]), f32(fr[1])
    t = time.time()
    r = track.track_pair(a, b, Config())
    fld = synth.uniform_strain(0.005 * k, 0.0, (128, 128), t=(0.8 * k, 0.0))
    gx, gy = synth.displacement(fld, n, n)
    save("pair_seq256", a=a, b=b, ux=r.ux, uy=r.uy, conf=r.conf, raw_ux=r.raw_ux, raw_uy=r.raw_uy, gt_ux=gx,
         gt_uy=gy, **{q: r.strain[q] for q in ("Exx", "Eyy", "Exy", "gmax", "vol")})
    print(f"  {time.time() - t:.1f} s")

    # a 224^2 miniature of the 2048^2 benchmark pair: affine strain (exx 0.01, eyy -0.004, gxy 0.006) plus a
    # 1.5 px sinusoid of wavelength 64 px, polygon ROI over the central 80 %, noise 0.01
    n = 224
    fld = AffineSine([[1.01, 0.003], [0.003, 0.996]], (n / 2, n / 2), amp=1.5, wavelength=64.0)
    roi = np.zeros((n, n), bool)
    roi[int(0.1 * n):int(0.9 * n) + 1, int(0.1 * n):int(0.9 * n) + 1] = True
    pair_case("pair_affsin", n, 7, fld, 0.01, roi=roi)

    # a dense guess (the init of a sequence leg): POC corrects it at the grid points
    n = 160
    fld = synth.uniform_strain(0.004, 0.002, (80, 80), t=(3.4, 2.8))
    yy, xx = np.mgrid[0:n, 0:n].astype(float)
    pair_case("pair_init", n, 31, fld, 0.005, init=(f32(3.0 + 0.003 * xx), f32(2.5 + 0.002 * yy)))


if __name__ == "__main__":
    main()
