"""CPU oracle of the learned coarse proposal (include/optflow_cuda_net.h): the same network in plain torch on the
CPU, float32, with autograd for the gradients.

TEST INFRASTRUCTURE: the checker of the network's CUDA kernels (forward, backward), never part of the engine. It
rounds to bfloat16 exactly where the kernels do (the normalised input, every layer's input activations and the
weights that enter the tensor-core GEMMs), so the forward passes differ only by the order of float32 accumulation.

Parameter layout (the flat float32 vector of ofc_net_param_count() values): per layer a [cout][kpad] weight matrix
(kpad = 9 cin rounded up to 16, column (ky * 3 + kx) * cin + c; the padding columns unused) followed by cout biases.
"""
import numpy as np
import torch
import torch.nn.functional as F

SPECS = [(1, 16, 2, 1, 1), (16, 32, 2, 1, 1), (32, 32, 2, 1, 1), (32, 32, 1, 1, 0),
         (160, 64, 1, 1, 1), (64, 64, 1, 2, 1), (64, 32, 1, 4, 1), (32, 16, 1, 1, 0)]
R = 5
D = 2 * R + 1
FEAT = 32
SCALE = 8


def kpad(cin):
    return (9 * cin + 15) // 16 * 16


def param_count():
    return sum(co * kpad(ci) + co for ci, co, *_ in SPECS)


def layer_offset(l):
    return sum(co * kpad(ci) + co for ci, co, *_ in SPECS[:l])


def unpack(params):
    """[(weight (cout, cin, 3, 3), bias (cout,))] from the flat vector (a torch tensor)."""
    out, o = [], 0
    for ci, co, *_ in SPECS:
        kp = kpad(ci)
        wm = params[o:o + co * kp].reshape(co, kp)[:, :9 * ci]
        o += co * kp
        b = params[o:o + co]
        o += co
        # column (ky 3 + kx) cin + c -> (cout, cin, ky, kx)
        out.append((wm.reshape(co, 3, 3, ci).permute(0, 3, 1, 2), b))
    return out


def init_params(seed=0):
    """He-initialised weights, zero biases, the padding columns zero (float32 numpy)."""
    rng = np.random.default_rng(seed)
    chunks = []
    for l, (ci, co, *_) in enumerate(SPECS):
        kp = kpad(ci)
        w = np.zeros((co, kp), np.float32)
        std = np.sqrt(2.0 / (9 * ci)) if l != len(SPECS) - 1 else 0.1 * np.sqrt(1.0 / (9 * ci))
        w[:, :9 * ci] = rng.normal(0.0, std, (co, 9 * ci))
        if l == len(SPECS) - 1:
            w[2:] = 0.0
        chunks += [w.ravel(), np.zeros(co, np.float32)]
    return np.concatenate(chunks)


def _bf(x):
    return x.to(torch.bfloat16).to(torch.float32)


def forward(params, i1, i2):
    """flow (nb, h/8, w/8, 2) of image batches i1, i2 (nb, h, w) float32 torch tensors."""
    layers = unpack(params)
    nb = i1.shape[0]
    x = torch.cat([i1, i2], 0)
    mean = x.double().mean(dim=(1, 2), keepdim=True)
    var = (x.double() ** 2).mean(dim=(1, 2), keepdim=True) - mean ** 2
    x = (x - mean.float()) * (1.0 / (var.clamp_min(0).sqrt() + 1e-6)).float()
    x = _bf(x)[:, None]
    for l in range(4):
        ci, co, s, d, relu = SPECS[l]
        w, b = layers[l]
        x = F.conv2d(_bf(x), _bf(w), b, stride=s, padding=d, dilation=d)
        if relu:
            x = F.relu(x)
    f = _bf(x)
    f1, f2 = f[:nb], f[nb:]
    h8, w8 = f1.shape[2:]
    pad = F.pad(f2, (R, R, R, R))
    corr = torch.stack([(f1 * pad[:, :, R + dy:R + dy + h8, R + dx:R + dx + w8]).sum(1) / FEAT
                        for dy in range(-R, R + 1) for dx in range(-R, R + 1)], 1)
    x = torch.cat([corr, f1, torch.zeros(nb, 160 - D * D - FEAT, h8, w8)], 1)
    for l in range(4, 8):
        ci, co, s, d, relu = SPECS[l]
        w, b = layers[l]
        x = F.conv2d(_bf(x), _bf(w), b, stride=s, padding=d, dilation=d)
        if relu:
            x = F.relu(x)
    p = torch.softmax(corr, 1)
    ks = torch.arange(D * D)
    dxs = (ks % D - R).float()[None, :, None, None]
    dys = (ks // D - R).float()[None, :, None, None]
    u = SCALE * (p * dxs).sum(1) + x[:, 0]
    v = SCALE * (p * dys).sum(1) + x[:, 1]
    return torch.stack([u, v], -1)


def loss_and_grads(params_np, i1, i2, target, mask):
    """(loss, flow, gradient) of the training loss: (1 / cells) sum over the masked cells of
    sqrt(|flow - target|^2 + 0.01)."""
    p = torch.tensor(params_np, dtype=torch.float32, requires_grad=True)
    flow = forward(p, torch.as_tensor(i1), torch.as_tensor(i2))
    t = torch.as_tensor(target)
    m = torch.as_tensor(mask).float()
    r = torch.sqrt(((flow - t) ** 2).sum(-1) + 0.01)
    loss = (r * m).sum() / m.numel()
    loss.backward()
    return float(loss.detach()), flow.detach().numpy(), p.grad.numpy().copy()
