"""The learned coarse proposal (include/optflow_cuda_net.h): the network object, its training pairs and its training.

The network predicts the displacement field at 1/8 resolution from an image pair; in an engine with
``Engine.set_coarse_net`` it replaces the POC coarse stage of pairs without a start field
(python/optflow_ref/poc.py:216-239, rust/crates/optflow-core/src/poc.rs:694 coarse_flow); the phase refinement always
follows, and tiles whose refined confidence fails fall back to POC. Forward, backward and the optimiser are the
library's own CUDA kernels (bfloat16 tensor-core GEMMs with float32 accumulation); torch supplies device memory and
streams only.

Training pairs (``training_pair``) are rendered by the engine's synthetic generator with known fields: a
Gaussian-process displacement (length scale 64-512 px, log-uniform; amplitude up to min(40, length / 8) px, so that
strains stay below about 15 %) plus a straight shear band (slip up to 4 px, width 4-16 px, random angle), speckle of
mean diameter 3-5 px, noise 0.003-0.02, 8 bits. A share of the pairs can take the plain method's own output (POC +
refine, where its confidence passes) as the target instead of the known field.
"""
import ctypes
import os

import numpy as np

from . import _abi, synth
from .config import Config

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "coarse_net.npz")
SCALE = 8
SPECS = [(1, 16), (16, 32), (32, 32), (32, 32), (160, 64), (64, 64), (64, 32), (32, 16)]  # (cin, cout) per layer


def param_count():
    return int(_abi.load().ofc_net_param_count())


def load_weights(path=WEIGHTS):
    """The trained parameters shipped with the package (float32 vector)."""
    with np.load(path) as z:
        return np.ascontiguousarray(z["params"], dtype=np.float32)


def init_params(seed):
    """He-initialised weights (the layer table of include/optflow_cuda_net.h), zero biases, padding columns zero."""
    rng = np.random.default_rng(seed)
    chunks = []
    for l, (ci, co) in enumerate(SPECS):
        kp = (9 * ci + 15) // 16 * 16
        wm = np.zeros((co, kp), np.float32)
        last = l == len(SPECS) - 1
        std = 0.1 * np.sqrt(1.0 / (9 * ci)) if last else np.sqrt(2.0 / (9 * ci))
        wm[:, :9 * ci] = rng.normal(0.0, std, (co, 9 * ci))
        if last:
            wm[2:] = 0.0  # only the first two output channels are used
        chunks += [wm.ravel(), np.zeros(co, np.float32)]
    return np.concatenate(chunks)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class CoarseNet:
    """A network on one CUDA device: parameters, Adam state and work buffers (ofc_net)."""

    def __init__(self, device=0, params=None):
        self.lib = _abi.load()
        err = ctypes.create_string_buffer(1024)
        h = self.lib.ofc_net_create(int(device), err, 1024)
        if not h:
            raise _abi.EngineError(2, err.value.decode())
        self.handle = ctypes.c_void_p(h)
        self.device = device
        if params is not None:
            self.set_params(params)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.ofc_net_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call(self, name, *args):
        err = ctypes.create_string_buffer(1024)
        st = getattr(self.lib, name)(self.handle, *args, err, 1024)
        if st != 0:
            raise _abi.EngineError(st, err.value.decode())

    def set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._call("ofc_net_set_params", p.ctypes.data_as(_abi.c_float_p), p.size)

    def get_params(self):
        p = np.empty(param_count(), np.float32)
        self._call("ofc_net_get_params", p.ctypes.data_as(_abi.c_float_p), p.size)
        return p

    @staticmethod
    def _stream(stream):
        import torch
        return ctypes.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)

    def forward(self, i1, i2, stream=None):
        """Flow (nb, h/8, w/8, 2) of CUDA float32 image batches i1, i2 (nb, h, w); h, w multiples of 8."""
        import torch
        nb, h, w = i1.shape
        flow = torch.empty((nb, h // SCALE, w // SCALE, 2), dtype=torch.float32, device=i1.device)
        self._call("ofc_net_forward", _ptr(i1), _ptr(i2), nb, h, w, _ptr(flow), self._stream(stream))
        return flow

    def gradients(self, i1, i2, target, mask, grads=None, stream=None):
        """(loss, flow, grads): forward and backward of the training loss on CUDA tensors; grads None: the network's
        own buffer, which adam() then reads."""
        import torch
        nb, h, w = i1.shape
        flow = torch.empty((nb, h // SCALE, w // SCALE, 2), dtype=torch.float32, device=i1.device)
        loss = ctypes.c_double()
        self._call("ofc_net_gradients", _ptr(i1), _ptr(i2), nb, h, w, _ptr(target), _ptr(mask), _ptr(flow),
                   _ptr(grads) if grads is not None else None, ctypes.byref(loss), self._stream(stream))
        return loss.value, flow, grads

    def adam(self, lr, grads=None, stream=None):
        self._call("ofc_net_adam", _ptr(grads) if grads is not None else None, ctypes.c_float(lr),
                   self._stream(stream))


# ---------------------------------------------------------------- training pairs
def random_field(rng, h, w):
    """A Gaussian-process displacement field plus a straight shear band (the training and held-out distribution)."""
    length = float(np.exp(rng.uniform(np.log(64.0), np.log(512.0))))
    amp = float(rng.uniform(0.0, min(40.0, length / 8.0)))
    grid, gx0, gy0 = synth.gp_grid(h, w, length, amp, rng)
    ang = rng.uniform(0, np.pi)
    band = synth.Band(e=(float(rng.uniform(0, w)), float(rng.uniform(0, h))), t=(float(np.cos(ang)), float(np.sin(ang))),
                      delta=float(rng.uniform(0.0, 4.0)), width=float(rng.uniform(4.0, 16.0)))
    return synth.Field(grid=grid, gx0=gx0, gy0=gy0, gh=16.0, bands=[band])


def cell_target(field, h, w):
    """The known displacement at the cell centres (8 i + 3.5) and the cells whose displaced centre stays 8 px inside
    the image."""
    ys = np.arange(h // SCALE) * SCALE + 3.5
    xs = np.arange(w // SCALE) * SCALE + 3.5
    X, Y = np.meshgrid(xs, ys)
    ux, uy = field.displacement_at(X, Y)
    tgt = np.stack([ux, uy], -1).astype(np.float32)
    xx, yy = X + ux, Y + uy
    mask = ((xx >= 8) & (xx < w - 8) & (yy >= 8) & (yy < h - 8)).astype(np.uint8)
    return tgt, mask


def training_pair(rng, h, w, engine=None):
    """(a, b, field): a seeded speckle pair (float32, 8-bit levels) under a random field."""
    field = random_field(rng, h, w)
    rmax = float(rng.uniform(2.0, 3.5))
    p = synth.make_pattern(h, w, seed=int(rng.integers(1 << 31)), rmin=1.5, rmax=rmax)
    noise = float(rng.uniform(0.003, 0.02))
    a = synth.degrade(synth.render(p, h, w, None, engine=engine), seed=int(rng.integers(1 << 31)), noise=noise, bits=8)
    b = synth.degrade(synth.render(p, h, w, field, engine=engine), seed=int(rng.integers(1 << 31)), noise=noise, bits=8)
    return a, b, field


def plain_target(a, b, engine, cfg=None):
    """The plain method's own result (POC + refine) at the cell centres, masked where its confidence fails."""
    from .api import track_pair
    cfg = cfg or Config()
    r = track_pair(a, b, cfg, engine=engine)
    h, w = a.shape
    ys = (np.arange(h // SCALE) * SCALE + 3).astype(int)
    xs = (np.arange(w // SCALE) * SCALE + 3).astype(int)
    u = 0.5 * (r.raw_ux[np.ix_(ys, xs)] + r.raw_ux[np.ix_(ys + 1, xs + 1)])
    v = 0.5 * (r.raw_uy[np.ix_(ys, xs)] + r.raw_uy[np.ix_(ys + 1, xs + 1)])
    ok = (r.conf[np.ix_(ys, xs)] >= cfg.conf_min) & np.isfinite(u) & np.isfinite(v)
    return np.stack([np.nan_to_num(u), np.nan_to_num(v)], -1).astype(np.float32), ok.astype(np.uint8)


def make_dataset(n, size, seed, engine=None, plain_share=0.0, log=None):
    """n training pairs of size x size: uint8 frames (n, 2, size, size), targets (n, size/8, size/8, 2) and masks."""
    rng = np.random.default_rng(seed)
    frames = np.empty((n, 2, size, size), np.uint8)
    tg = np.empty((n, size // SCALE, size // SCALE, 2), np.float32)
    mk = np.empty((n, size // SCALE, size // SCALE), np.uint8)
    for i in range(n):
        a, b, field = training_pair(rng, size, size, engine)
        frames[i, 0] = np.round(a * 255)
        frames[i, 1] = np.round(b * 255)
        if plain_share > 0 and rng.random() < plain_share:
            tg[i], mk[i] = plain_target(a, b, engine)
        else:
            tg[i], mk[i] = cell_target(field, size, size)
        if log and (i + 1) % 2000 == 0:
            log(f"{i + 1} / {n} training pairs")
    return frames, tg, mk


def train(frames, targets, masks, steps, batch=16, lr=1e-3, seed=0, params=None, device=0, log=None):
    """Adam on the network's own kernels over the dataset (uint8 frames), cosine decay of the learning rate; returns
    (parameters, losses)."""
    import torch
    dev = torch.device("cuda", device)
    net = CoarseNet(device, init_params(seed) if params is None else params)
    fr = torch.as_tensor(frames).to(dev)
    tg = torch.as_tensor(targets).to(dev)
    mk = torch.as_tensor(masks).to(dev)
    n = fr.shape[0]
    g = torch.Generator(device="cpu").manual_seed(seed)
    stream = torch.cuda.current_stream(dev)
    losses = []
    for s in range(steps):
        idx = torch.randint(0, n, (batch,), generator=g).to(dev)
        x = fr[idx].float() / 255.0
        i1, i2 = x[:, 0].contiguous(), x[:, 1].contiguous()
        loss, _, _ = net.gradients(i1, i2, tg[idx].contiguous(), mk[idx].contiguous(), stream=stream)
        net.adam(lr * 0.5 * (1.0 + np.cos(np.pi * s / steps)), stream=stream)
        losses.append(loss)
        if log and (s + 1) % 500 == 0:
            log(f"step {s + 1}: loss {np.mean(losses[-500:]):.4f}")
    return net.get_params(), losses


def time_net(size, batch, reps):
    """Device time (CUDA events, median) of the forward pass on one size x size pair, and of one training step
    (forward, backward, Adam) on `batch` pairs of 256^2; prints one JSON line."""
    import json
    import torch
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(5)
    net = CoarseNet(0, init_params(1))
    a, b, _ = training_pair(rng, size, size)
    d_a, d_b = torch.from_numpy(a)[None].to(dev), torch.from_numpy(b)[None].to(dev)
    stream = torch.cuda.current_stream(dev)

    def timed(fn):
        fn()
        ms = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ms.append(e0.elapsed_time(e1))
        return float(np.median(ms))

    fwd = timed(lambda: net.forward(d_a, d_b, stream=stream))
    fr = [training_pair(rng, 256, 256) for _ in range(batch)]
    i1 = torch.from_numpy(np.stack([f[0] for f in fr])).to(dev)
    i2 = torch.from_numpy(np.stack([f[1] for f in fr])).to(dev)
    tg = torch.zeros((batch, 32, 32, 2), dtype=torch.float32, device=dev)
    mk = torch.ones((batch, 32, 32), dtype=torch.uint8, device=dev)

    def step():
        net.gradients(i1, i2, tg, mk, stream=stream)
        net.adam(1e-4, stream=stream)

    trn = timed(step)
    print(json.dumps({"forward_ms": fwd, "size": size, "train_step_ms": trn, "batch": batch, "train_size": 256}))


def main(argv=None):
    """python -m optflow_b200.net train [--pairs N] [--size S] [--steps K] [--batch B] [--seed S] [--out PATH]:
    renders the training set on the GPU, trains on it with the network's kernels and writes the parameters."""
    import argparse
    import time
    ap = argparse.ArgumentParser(prog="python -m optflow_b200.net")
    ap.add_argument("cmd", choices=["train", "time"])
    ap.add_argument("--pairs", type=int, default=20000)
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--plain-share", type=float, default=0.1)
    ap.add_argument("--seed", type=int, default=23)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--reps", type=int, default=20)
    a = ap.parse_args(argv)
    if a.cmd == "time":
        time_net(a.size, a.batch, a.reps)
        return
    from .api import Engine
    log = lambda m: print(f"[{time.strftime('%H:%M:%S')}] {m}", flush=True)
    eng = Engine(0)
    t0 = time.time()
    frames, tg, mk = make_dataset(a.pairs, a.size, a.seed, engine=eng, plain_share=a.plain_share, log=log)
    log(f"dataset: {a.pairs} pairs of {a.size}^2 in {time.time() - t0:.1f} s")
    t0 = time.time()
    params, losses = train(frames, tg, mk, a.steps, batch=a.batch, lr=a.lr, seed=a.seed, log=log)
    log(f"training: {a.steps} steps of {a.batch} pairs in {time.time() - t0:.1f} s, final loss "
        f"{np.mean(losses[-500:]):.4f}")
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    np.savez_compressed(a.out, params=params, losses=np.asarray(losses, np.float32),
                        meta=np.array(f"pairs={a.pairs} size={a.size} steps={a.steps} batch={a.batch} lr={a.lr} "
                                      f"plain_share={a.plain_share} seed={a.seed}"))
    log(f"wrote {a.out}")


if __name__ == "__main__":
    main()
