"""CPU restatement of the learned warm start's CNN arithmetic (test infrastructure only).

The reference has no learned component, so there is nothing of the reference to pin this
against; its own backward pass is pinned by a central finite-difference check in float64
(tests/test_cnn_oracle.py).  With `exact=False` it mirrors the device network's rounding
points: every stored activation and gradient tensor is rounded to bfloat16 (round to
nearest even), products are accumulated in float64 (the device accumulates in float32, so
tests compare with a tolerance), pooling / upsampling sums use the device's float32
order ((a + b) + (c + d)).

Layouts follow the device: activations NHWC, weights w[tap][cout][cin] with
tap = 3 * (dy + 1) + (dx + 1), the input sampled at (y + dy, x + dx), zero padding.
"""
from __future__ import annotations

import numpy as np

LAYERS = [
    ("c0a", 2, 32), ("c0b", 32, 32),
    ("c1a", 32, 64), ("c1b", 64, 64),
    ("c2a", 64, 128), ("c2b", 128, 128),
    ("c3a", 128, 256), ("c3b", 256, 256),
    ("d2", 384, 128), ("d1", 192, 64), ("d0", 96, 32),
    ("head", 32, 2),
]


def bf16(x):
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = (a + np.uint32(0x7FFF) + ((a >> np.uint32(16)) & np.uint32(1))) & np.uint32(0xFFFF0000)
    return r.view(np.float32)


def _shift(x, dy, dx):
    """x sampled at (y + dy, x + dx) with zeros outside."""
    n, H, W, C = x.shape
    out = np.zeros_like(x)
    ys, yd = (slice(dy, H), slice(0, H - dy)) if dy >= 0 else (slice(0, H + dy), slice(-dy, H))
    xs, xd = (slice(dx, W), slice(0, W - dx)) if dx >= 0 else (slice(0, W + dx), slice(-dx, W))
    out[:, yd, xd] = x[:, ys, xs]
    return out


def conv3x3(x, w9, bias=None):
    """y[p][co] = sum_tap sum_ci x[p + tap][ci] w9[tap][co][ci] (+ bias), float64."""
    x = np.asarray(x, np.float64)
    w9 = np.asarray(w9, np.float64)
    y = np.zeros(x.shape[:3] + (w9.shape[1],), np.float64)
    for t in range(9):
        y += _shift(x, t // 3 - 1, t % 3 - 1) @ w9[t].T
    if bias is not None:
        y += np.asarray(bias, np.float64)
    return y


def conv3x3_dgrad(dy, w9):
    """dx[p][ci] = sum_tap sum_co dy[p - tap][co] w9[tap][co][ci]."""
    dy = np.asarray(dy, np.float64)
    w9 = np.asarray(w9, np.float64)
    dx = np.zeros(dy.shape[:3] + (w9.shape[2],), np.float64)
    for t in range(9):
        dx += _shift(dy, -(t // 3 - 1), -(t % 3 - 1)) @ w9[t]
    return dx


def conv3x3_wgrad(x, dy):
    """dw[tap][co][ci] = sum_p dy[p][co] x[p + tap][ci]."""
    x = np.asarray(x, np.float64)
    dy = np.asarray(dy, np.float64)
    C = x.shape[3]
    g = dy.reshape(-1, dy.shape[3])
    return np.stack([g.T @ _shift(x, t // 3 - 1, t % 3 - 1).reshape(-1, C) for t in range(9)])


def avgpool2(x):
    x = np.asarray(x, np.float32)
    s = (x[:, 0::2, 0::2] + x[:, 0::2, 1::2]) + (x[:, 1::2, 0::2] + x[:, 1::2, 1::2])
    return s * np.float32(0.25)


def avgpool2_bwd(dy):
    g = np.asarray(dy, np.float32) * np.float32(0.25)
    return np.repeat(np.repeat(g, 2, axis=1), 2, axis=2)


def upsample2(x):
    return np.repeat(np.repeat(np.asarray(x), 2, axis=1), 2, axis=2)


def upsample2_bwd(dy):
    d = np.asarray(dy, np.float32)
    return (d[:, 0::2, 0::2] + d[:, 0::2, 1::2]) + (d[:, 1::2, 0::2] + d[:, 1::2, 1::2])


def flow_mse(pred, label):
    """loss = sum |pred - label|^2 / (2P); dpred = (pred - label) / P (float32 ops)."""
    pred = np.asarray(pred, np.float32)
    label = np.asarray(label, np.float32)
    P = pred.shape[0] * pred.shape[1] * pred.shape[2]
    d = pred - label
    loss = float(np.sum((d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]).astype(np.float64)) / (2.0 * P))
    return loss, d * np.float32(1.0 / np.float32(P))


def adam(w, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    f = np.float32
    b1, b2, lr, eps = f(b1), f(b2), f(lr), f(eps)
    bc1, bc2 = f(1.0 - b1.astype(np.float64) ** step), f(1.0 - b2.astype(np.float64) ** step)
    m = b1 * m + (f(1) - b1) * g
    v = b2 * v + (f(1) - b2) * (g * g)
    w = w - (lr * (m / bc1)) / (np.sqrt(v / bc2) + eps)
    return w.astype(np.float32), m.astype(np.float32), v.astype(np.float32)


class Net:
    """The warm-start network on the CPU: params[name] = (w9 [9][co][ci], bias [co])."""

    def __init__(self, params, exact=False):
        self.p = params
        self.exact = exact

    def _r(self, x):
        return np.asarray(x, np.float64) if self.exact else bf16(np.asarray(x, np.float32))

    def _conv(self, name, x, relu=True):
        w, b = self.p[name]
        if not self.exact:
            w = bf16(w)
        y = conv3x3(x, w, b)
        return np.maximum(y, 0.0) if relu else y

    def forward(self, x0):
        """x0 (n, S, S, 2) -> flow (n, S, S, 2); keeps the activations for backward()."""
        r, c = self._r, self._conv
        a = {"x0": r(x0)}
        a["a0"] = r(c("c0a", a["x0"]))
        a["e0"] = r(c("c0b", a["a0"]))
        a["p1"] = r(avgpool2(a["e0"])) if not self.exact else self._pool(a["e0"])
        a["a1"] = r(c("c1a", a["p1"]))
        a["e1"] = r(c("c1b", a["a1"]))
        a["p2"] = r(avgpool2(a["e1"])) if not self.exact else self._pool(a["e1"])
        a["a2"] = r(c("c2a", a["p2"]))
        a["e2"] = r(c("c2b", a["a2"]))
        a["p3"] = r(avgpool2(a["e2"])) if not self.exact else self._pool(a["e2"])
        a["a3"] = r(c("c3a", a["p3"]))
        a["e3"] = r(c("c3b", a["a3"]))
        a["cat2"] = np.concatenate([upsample2(a["e3"]), a["e2"]], axis=3)
        a["d2"] = r(c("d2", a["cat2"]))
        a["cat1"] = np.concatenate([upsample2(a["d2"]), a["e1"]], axis=3)
        a["d1"] = r(c("d1", a["cat1"]))
        a["cat0"] = np.concatenate([upsample2(a["d1"]), a["e0"]], axis=3)
        a["d0"] = r(c("d0", a["cat0"]))
        out = c("head", a["d0"], relu=False)
        a["out"] = out if self.exact else out.astype(np.float32)
        self.a = a
        return a["out"]

    @staticmethod
    def _pool(x):
        return 0.25 * (x[:, 0::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 0::2] + x[:, 1::2, 1::2])

    def backward(self, dout):
        """dout (n, S, S, 2) -> {name: (dw, db)} in float64."""
        a, r, ex = self.a, self._r, self.exact
        grads = {}

        def wb(name):
            w = self.p[name][0]
            return w if ex else bf16(w)

        def layer(name, x, dy):
            grads[name] = (conv3x3_wgrad(x, dy), np.asarray(dy, np.float64).sum(axis=(0, 1, 2)))
            return conv3x3_dgrad(dy, wb(name))

        def relu(g, y):
            return np.where(np.asarray(y) > 0, g, 0.0)

        def pool_bwd(g):
            return avgpool2_bwd(g) if not ex else np.repeat(np.repeat(0.25 * g, 2, axis=1), 2, axis=2)

        def up_bwd(g):
            return upsample2_bwd(g) if not ex else (g[:, 0::2, 0::2] + g[:, 0::2, 1::2] + g[:, 1::2, 0::2] +
                                                    g[:, 1::2, 1::2])

        g = r(dout)
        g = relu(r(layer("head", a["d0"], g)), a["d0"])
        gc0 = r(layer("d0", a["cat0"], g))
        g = relu(r(up_bwd(gc0[..., :64])), a["d1"])
        gc1 = r(layer("d1", a["cat1"], g))
        g = relu(r(up_bwd(gc1[..., :128])), a["d2"])
        gc2 = r(layer("d2", a["cat2"], g))
        g = relu(r(up_bwd(gc2[..., :256])), a["e3"])
        g = relu(r(layer("c3b", a["a3"], g)), a["a3"])
        gp3 = r(layer("c3a", a["p3"], g))
        g = relu(r(np.asarray(pool_bwd(gp3), np.float32 if not ex else np.float64) + gc2[..., 256:]), a["e2"])
        g = relu(r(layer("c2b", a["a2"], g)), a["a2"])
        gp2 = r(layer("c2a", a["p2"], g))
        g = relu(r(np.asarray(pool_bwd(gp2), np.float32 if not ex else np.float64) + gc1[..., 128:]), a["e1"])
        g = relu(r(layer("c1b", a["a1"], g)), a["a1"])
        gp1 = r(layer("c1a", a["p1"], g))
        g = relu(r(np.asarray(pool_bwd(gp1), np.float32 if not ex else np.float64) + gc0[..., 64:]), a["e0"])
        g = relu(r(layer("c0b", a["a0"], g)), a["a0"])
        layer("c0a", a["x0"], g)
        return grads


def init_params(seed=0):
    """Same initialisation as the device network (He normal, zero bias)."""
    rng = np.random.default_rng(seed)
    p = {}
    for name, ci, co in LAYERS:
        std = np.sqrt(2.0 / (9 * ci)) if name != "head" else np.sqrt(1.0 / (9 * ci))
        w = rng.normal(0.0, std, 9 * co * ci).astype(np.float32).reshape(9, co, ci)
        p[name] = (w, np.zeros(co, np.float32))
    return p


def flat_to_params(flat):
    p, o = {}, 0
    for name, ci, co in LAYERS:
        w = np.asarray(flat[o:o + 9 * co * ci], np.float32).reshape(9, co, ci)
        o += 9 * co * ci
        b = np.asarray(flat[o:o + co], np.float32)
        o += co
        p[name] = (w, b)
    return p
