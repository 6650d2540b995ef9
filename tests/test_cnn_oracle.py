"""The CNN oracle's backward pass against central finite differences (float64), and the
bfloat16 rounding helper against torch's conversion."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import cnn_oracle as C  # noqa: E402


def _loss(net, x, R):
    return float(np.sum(net.forward(x) * R))


@pytest.mark.parametrize("layer", ["c0a", "c1b", "c3b", "d2", "d0", "head"])
def test_backward_matches_finite_differences(layer):
    rng = np.random.default_rng(1)
    p = C.init_params(3)
    p = {k: (w.astype(np.float64), rng.normal(0, 0.1, b.shape)) for k, (w, b) in p.items()}
    net = C.Net(p, exact=True)
    x = rng.uniform(0, 1, (1, 16, 16, 2))
    R = rng.normal(0, 1, (1, 16, 16, 2))
    net.forward(x)
    g = net.backward(R)
    w, b = p[layer]
    eps = 1e-6
    for idx in [tuple(rng.integers(0, s) for s in w.shape) for _ in range(4)]:
        old = w[idx]
        w[idx] = old + eps
        lp = _loss(net, x, R)
        w[idx] = old - eps
        lm = _loss(net, x, R)
        w[idx] = old
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[layer][0][idx]) <= 1e-5 * max(1.0, abs(fd)), (layer, idx, fd, g[layer][0][idx])
    j = int(rng.integers(0, b.shape[0]))
    old = b[j]
    b[j] = old + eps
    lp = _loss(net, x, R)
    b[j] = old - eps
    lm = _loss(net, x, R)
    b[j] = old
    assert abs((lp - lm) / (2 * eps) - g[layer][1][j]) <= 1e-5 * max(1.0, abs(g[layer][1][j]))


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(0, 1, 10000), rng.normal(0, 1e-3, 1000), [0.0, -0.0, 1.0, 65504.0]]).astype(np.float32)
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(C.bf16(x), want)


def test_dgrad_is_adjoint_of_conv():
    rng = np.random.default_rng(2)
    x = rng.normal(0, 1, (2, 8, 8, 5))
    w = rng.normal(0, 1, (9, 7, 5))
    dy = rng.normal(0, 1, (2, 8, 8, 7))
    lhs = np.sum(C.conv3x3(x, w) * dy)
    rhs = np.sum(x * C.conv3x3_dgrad(dy, w))
    assert abs(lhs - rhs) < 1e-9 * abs(lhs)
    gw = C.conv3x3_wgrad(x, dy)
    assert abs(np.sum(gw * w) - lhs) < 1e-9 * abs(lhs)
