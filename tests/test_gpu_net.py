"""The learned coarse proposal's CUDA kernels (include/optflow_cuda_net.h) against the CPU oracle of the same
network (oracle/coarse_net.py: plain torch on the CPU, float32 autograd, bfloat16 rounding where the kernels round).

Bars: the loss within 1e-3 (relative), the flow within 2e-2 px, every layer's weight and bias gradient within 3e-2
of the oracle's in relative L2 norm (the kernels round the backward activation gradients to bfloat16 before the
tensor-core GEMMs; the oracle keeps them in float32)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(nb, h, w, seed):
    from optflow_b200 import net
    rng = np.random.default_rng(seed)
    i1, i2, tg, mk = [], [], [], []
    for _ in range(nb):
        a, b, f = net.training_pair(rng, h, w)
        t, m = net.cell_target(f, h, w)
        i1.append(a)
        i2.append(b)
        tg.append(t)
        mk.append(m)
    return np.stack(i1), np.stack(i2), np.stack(tg), np.stack(mk)


@pytest.mark.parametrize("seed", [0, 1])
def test_net_gradients_match_the_cpu_oracle(seed):
    import torch
    import coarse_net
    from optflow_b200 import net
    assert coarse_net.param_count() == net.param_count()
    params = coarse_net.init_params(seed)
    i1, i2, tg, mk = _batch(2, 96, 128, seed)
    want_loss, want_flow, want_g = coarse_net.loss_and_grads(params, i1, i2, tg, mk)
    dev = torch.device("cuda")
    m = net.CoarseNet(0, params)
    grads = torch.empty(params.size, dtype=torch.float32, device=dev)
    t = lambda a: torch.as_tensor(a).to(dev).contiguous()
    loss, flow, _ = m.gradients(t(i1), t(i2), t(tg), t(mk), grads=grads)
    torch.cuda.synchronize()
    assert abs(loss - want_loss) < 1e-3 * abs(want_loss), (loss, want_loss)
    assert np.abs(flow.cpu().numpy() - want_flow).max() < 2e-2
    g = grads.cpu().numpy()
    for l, (ci, co, *_) in enumerate(coarse_net.SPECS):
        o = coarse_net.layer_offset(l)
        n = co * coarse_net.kpad(ci) + co
        a, b = g[o:o + n], want_g[o:o + n]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert rel < 3e-2, (l, rel)


def test_net_forward_equals_the_gradient_pass_and_training_lowers_the_loss():
    import torch
    from optflow_b200 import net
    i1, i2, tg, mk = _batch(4, 128, 128, 5)
    dev = torch.device("cuda")
    t = lambda a: torch.as_tensor(a).to(dev).contiguous()
    m = net.CoarseNet(0, net.init_params(3))
    f0 = m.forward(t(i1), t(i2))
    l0, f1, _ = m.gradients(t(i1), t(i2), t(tg), t(mk))
    assert torch.equal(f0, f1)
    for _ in range(30):
        m.gradients(t(i1), t(i2), t(tg), t(mk))
        m.adam(2e-3)
    l1, _, _ = m.gradients(t(i1), t(i2), t(tg), t(mk))
    assert l1 < 0.7 * l0, (l0, l1)
