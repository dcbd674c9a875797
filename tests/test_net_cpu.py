"""The learned coarse proposal without a GPU: the parameter layout the library declares, the oracle's and the
package's initialisation agree, and the oracle network (oracle/coarse_net.py) is consistent: its soft-argmax prior
recovers a pure shift of the features, and its autograd gradient matches central differences on a few weights."""
import numpy as np
import torch

import coarse_net
from optflow_b200 import net


def test_parameter_layout():
    assert coarse_net.param_count() == net.param_count()
    np.testing.assert_array_equal(coarse_net.init_params(3), net.init_params(3))


def test_oracle_gradient_matches_central_differences():
    """The flow is affine in the last layer's two used biases (they enter after every bfloat16 rounding), so central
    differences of the loss in them are exact up to float32 rounding."""
    rng = np.random.default_rng(0)
    p = coarse_net.init_params(1)
    i1 = rng.random((1, 48, 48)).astype(np.float32)
    i2 = np.roll(i1, (2, -3), (1, 2))
    t = rng.normal(0, 2, (1, 6, 6, 2)).astype(np.float32)
    m = np.ones((1, 6, 6), np.uint8)
    _, _, g = coarse_net.loss_and_grads(p, i1, i2, t, m)
    for k in (coarse_net.layer_offset(8) - 16, coarse_net.layer_offset(8) - 15):
        e = np.zeros_like(p)
        e[k] = 1e-2
        lp, _, _ = coarse_net.loss_and_grads(p + e, i1, i2, t, m)
        lm, _, _ = coarse_net.loss_and_grads(p - e, i1, i2, t, m)
        fd = (lp - lm) / 2e-2
        assert abs(fd - g[k]) < 1e-3 * max(1.0, abs(fd)), (k, fd, g[k])
