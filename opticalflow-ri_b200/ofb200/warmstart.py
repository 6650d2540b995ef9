"""Learned warm start for the 1024^2 Liu-Shen refinement.

The plain pipeline (Farneback at 512^2 and 1024^2, each followed by 60 Liu-Shen sweeps)
spends most of its time getting a good initial field for the last Liu-Shen solve.  Here an
encoder-decoder CNN maps a pyramid level's frame pair (the bicubic downsample by `factor`,
each frame divided by its maximum; the packaged weights run at 128^2 for 1024^2 frames) to
a flow at that level; one fused bilinear upsample turns it into the initial field of a
short full-size stage (one Farneback iteration and a few Liu-Shen sweeps for the packaged
calibration).  The solve's last update norm (its convergence residual) decides the result:
above a threshold calibrated on held-out pairs, the pair falls back to the plain pyramid.

Network (bf16 NHWC activations, f32 accumulation; ~1.75 M parameters):

    enc0  conv 2->32, conv 32->32        (S)      e0 -> cat0[64:96]
    enc1  pool, conv 32->64, conv 64->64 (S/2)    e1 -> cat1[128:192]
    enc2  pool, conv 64->128, 128->128   (S/4)    e2 -> cat2[256:384]
    enc3  pool, conv 128->256, 256->256  (S/8)    e3
    dec2  up(e3) | e2 -> conv 384->128   (S/4)
    dec1  up(d2) | e1 -> conv 192->64    (S/2)
    dec0  up(d1) | e0 -> conv 96->32     (S)
    head  conv 32->2 (f32, no ReLU)

All 3x3 convolutions with ReLU except the head; pooling is 2x2 average, upsampling nearest.
Every convolution runs on the tensor cores: forward and input gradient through
of_cnn_conv3x3, weight gradient through of_cnn_conv3x3_wgrad_tc; pooling and the rest
through the other of_cnn_* entry points.  torch provides device memory and the stream only.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from . import ops
from ._lib import call

__all__ = ["LAYERS", "WarmStartNet", "LearnedLiuShen", "LearnedBatch", "load_trained", "n_params"]

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "warmstart_weights.npz")

LAYERS = [  # name, cin, cout
    ("c0a", 2, 32), ("c0b", 32, 32),
    ("c1a", 32, 64), ("c1b", 64, 64),
    ("c2a", 64, 128), ("c2b", 128, 128),
    ("c3a", 128, 256), ("c3b", 256, 256),
    ("d2", 384, 128), ("d1", 192, 64), ("d0", 96, 32),
    ("head", 32, 2),
]
IN_CH = 16  # the 2 input channels padded to the tensor-core K granularity
RELU, F32 = 1, 2


def _pad16(c):
    return (c + 15) // 16 * 16


def _cin_pad(cin):
    return IN_CH if cin == 2 else cin


def n_params():
    return sum(9 * ci * co + co for _, ci, co in LAYERS)


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _sp():
    return ops.stream_ptr()


class WarmStartNet:
    """Parameters (f32 master copy, Adam state) and the forward / backward passes."""

    def __init__(self, seed=0, device="cuda"):
        self.device = torch.device(device)
        self.off = {}
        o = 0
        for name, ci, co in LAYERS:
            self.off[name] = (o, o + 9 * co * ci, ci, co)  # weights [9][co][ci], then bias [co]
            o += 9 * co * ci + co
        self.total = o
        rng = np.random.default_rng(seed)
        host = np.zeros(o, np.float32)
        for name, ci, co in LAYERS:
            wo, bo, _, _ = self.off[name]
            std = np.sqrt(2.0 / (9 * ci)) if name != "head" else np.sqrt(1.0 / (9 * ci))
            host[wo:bo] = rng.normal(0.0, std, 9 * co * ci).astype(np.float32)
        self.params = torch.from_numpy(host).to(self.device)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step_count = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.wf, self.wb = {}, {}
        for name, ci, co in LAYERS:
            self.wf[name] = torch.empty((9, _pad16(co), _cin_pad(ci)), dtype=torch.bfloat16, device=self.device)
            self.wb[name] = torch.empty((9, _cin_pad(ci), _pad16(co)), dtype=torch.bfloat16, device=self.device)
        self._bufs = {}
        self.pack()

    # ------------------------------------------------------------------ parameters
    def pack(self):
        """bf16 forward and input-gradient operands from the master weights."""
        for name, ci, co in LAYERS:
            wo, _, _, _ = self.off[name]
            w = ctypes.c_void_p(self.params.data_ptr() + 4 * wo)
            call("of_cnn_pack_weights", w, co, ci, _pad16(co), _cin_pad(ci), 0, _p(self.wf[name]), _sp())
            if name != "c0a":
                call("of_cnn_pack_weights", w, co, ci, _pad16(co), _cin_pad(ci), 1, _p(self.wb[name]), _sp())

    def _bias(self, name):
        return ctypes.c_void_p(self.params.data_ptr() + 4 * self.off[name][1])

    def _gw(self, name):
        return ctypes.c_void_p(self.grads.data_ptr() + 4 * self.off[name][0])

    def _gb(self, name):
        return ctypes.c_void_p(self.grads.data_ptr() + 4 * self.off[name][1])

    def adam(self, lr, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        call("of_cnn_adam", _p(self.params), _p(self.grads), _p(self.m), _p(self.v), self.total, float(lr), float(b1),
             float(b2), float(eps), self.step_count, _sp())
        self.pack()

    def state(self):
        return {"params": self.params.cpu().numpy(), "layers": np.array([f"{n}:{a}:{b}" for n, a, b in LAYERS])}

    def save(self, path):
        np.savez(path, **self.state())

    def load(self, path):
        d = np.load(path)
        if list(d["layers"]) != [f"{n}:{a}:{b}" for n, a, b in LAYERS]:
            raise ValueError(f"{path}: layer table does not match")
        self.params.copy_(torch.from_numpy(d["params"].astype(np.float32)))
        self.pack()
        return self

    # ------------------------------------------------------------------ buffers
    def buffers(self, n, S):
        key = (n, S)
        b = self._bufs.get(key)
        if b is not None:
            return b
        if S % 8 or S < 16:
            raise ValueError("input size must be a multiple of 8 and >= 16")
        bf = dict(dtype=torch.bfloat16, device=self.device)
        s1, s2, s3 = S // 2, S // 4, S // 8
        b = {
            "x0": torch.zeros((n, S, S, IN_CH), **bf),
            "a0": torch.empty((n, S, S, 32), **bf), "cat0": torch.empty((n, S, S, 96), **bf),
            "p1": torch.empty((n, s1, s1, 32), **bf), "a1": torch.empty((n, s1, s1, 64), **bf),
            "cat1": torch.empty((n, s1, s1, 192), **bf),
            "p2": torch.empty((n, s2, s2, 64), **bf), "a2": torch.empty((n, s2, s2, 128), **bf),
            "cat2": torch.empty((n, s2, s2, 384), **bf),
            "p3": torch.empty((n, s3, s3, 128), **bf), "a3": torch.empty((n, s3, s3, 256), **bf),
            "e3": torch.empty((n, s3, s3, 256), **bf),
            "d2": torch.empty((n, s2, s2, 128), **bf), "d1": torch.empty((n, s1, s1, 64), **bf),
            "d0": torch.empty((n, S, S, 32), **bf),
            "out": torch.empty((n, S, S, 2), dtype=torch.float32, device=self.device),
            "max2": torch.zeros((n, 2), dtype=torch.int32, device=self.device),
        }
        self._bufs[key] = b
        return b

    def grad_buffers(self, n, S):
        key = ("g", n, S)
        g = self._bufs.get(key)
        if g is not None:
            return g
        bf = dict(dtype=torch.bfloat16, device=self.device)
        s1, s2, s3 = S // 2, S // 4, S // 8
        g = {
            "dout": torch.zeros((n, S, S, 16), **bf),
            "d0": torch.empty((n, S, S, 32), **bf), "cat0": torch.empty((n, S, S, 96), **bf),
            "d1": torch.empty((n, s1, s1, 64), **bf), "cat1": torch.empty((n, s1, s1, 192), **bf),
            "d2": torch.empty((n, s2, s2, 128), **bf), "cat2": torch.empty((n, s2, s2, 384), **bf),
            "e3": torch.empty((n, s3, s3, 256), **bf), "a3": torch.empty((n, s3, s3, 256), **bf),
            "p3": torch.empty((n, s3, s3, 128), **bf), "a2": torch.empty((n, s2, s2, 128), **bf),
            "p2": torch.empty((n, s2, s2, 64), **bf), "a1": torch.empty((n, s1, s1, 64), **bf),
            "p1": torch.empty((n, s1, s1, 32), **bf), "a0": torch.empty((n, S, S, 32), **bf),
            "loss": torch.zeros((), dtype=torch.float64, device=self.device),
        }
        self._bufs[key] = g
        return g

    # ------------------------------------------------------------------ passes
    def _conv(self, name, x, xct, xco, cin, n, H, W, y, yct, yco, flags=RELU, cout_store=None, backward=False):
        ci, co = self.off[name][2], self.off[name][3]
        if backward:  # input gradient: y (cin channels) = conv(dy (cout_pad channels), flipped W^T)
            w, cout, store, bias = self.wb[name], _cin_pad(ci), cout_store or ci, None
        else:
            w, cout, store, bias = self.wf[name], _pad16(co), cout_store or co, self._bias(name)
        call("of_cnn_conv3x3", _p(x), n, H, W, cin, xct, xco, _p(w), cout, bias, flags, _p(y), yct, yco, store,
             _p(self.err), _sp())

    def pack_input(self, b, i, I0, I1):
        """Pair i of the batch: two f32 planes -> x0[i] (channels 0, 1)."""
        H, W = I0.shape
        x = b["x0"]
        call("of_cnn_pack_pair", _p(I0), _p(I1), H, W, I0.stride(0),
             ctypes.c_void_p(b["max2"].data_ptr() + 8 * i), ctypes.c_void_p(x.data_ptr() + 2 * i * H * W * IN_CH),
             IN_CH, _sp())

    def forward(self, b):
        n, S = b["x0"].shape[0], b["x0"].shape[1]
        s1, s2, s3 = S // 2, S // 4, S // 8
        cv = self._conv
        cv("c0a", b["x0"], IN_CH, 0, IN_CH, n, S, S, b["a0"], 32, 0)
        cv("c0b", b["a0"], 32, 0, 32, n, S, S, b["cat0"], 96, 64)
        call("of_cnn_avgpool2", _p(b["cat0"]), 96, 64, n, S, S, 32, _p(b["p1"]), 32, 0, _sp())
        cv("c1a", b["p1"], 32, 0, 32, n, s1, s1, b["a1"], 64, 0)
        cv("c1b", b["a1"], 64, 0, 64, n, s1, s1, b["cat1"], 192, 128)
        call("of_cnn_avgpool2", _p(b["cat1"]), 192, 128, n, s1, s1, 64, _p(b["p2"]), 64, 0, _sp())
        cv("c2a", b["p2"], 64, 0, 64, n, s2, s2, b["a2"], 128, 0)
        cv("c2b", b["a2"], 128, 0, 128, n, s2, s2, b["cat2"], 384, 256)
        call("of_cnn_avgpool2", _p(b["cat2"]), 384, 256, n, s2, s2, 128, _p(b["p3"]), 128, 0, _sp())
        cv("c3a", b["p3"], 128, 0, 128, n, s3, s3, b["a3"], 256, 0)
        cv("c3b", b["a3"], 256, 0, 256, n, s3, s3, b["e3"], 256, 0)
        call("of_cnn_upsample2", _p(b["e3"]), 256, 0, n, s3, s3, 256, _p(b["cat2"]), 384, 0, _sp())
        cv("d2", b["cat2"], 384, 0, 384, n, s2, s2, b["d2"], 128, 0)
        call("of_cnn_upsample2", _p(b["d2"]), 128, 0, n, s2, s2, 128, _p(b["cat1"]), 192, 0, _sp())
        cv("d1", b["cat1"], 192, 0, 192, n, s1, s1, b["d1"], 64, 0)
        call("of_cnn_upsample2", _p(b["d1"]), 64, 0, n, s1, s1, 64, _p(b["cat0"]), 96, 0, _sp())
        cv("d0", b["cat0"], 96, 0, 96, n, S, S, b["d0"], 32, 0)
        cv("head", b["d0"], 32, 0, 32, n, S, S, b["out"], 2, 0, flags=F32, cout_store=2)
        return b["out"]

    def loss(self, b, g, label, with_grad=True):
        """Mean squared flow error against label (n, S, S, 2) f32; dout for backward()."""
        n, S = b["x0"].shape[0], b["x0"].shape[1]
        g["loss"].zero_()
        call("of_cnn_flow_mse", _p(b["out"]), _p(label), n * S * S, _p(g["dout"]) if with_grad else None, 16,
             _p(g["loss"]), _sp())
        return g["loss"]

    def _wgrad(self, name, x, xct, xco, dy, dct, dco, n, H, W):
        _, _, ci, co = self.off[name]
        call("of_cnn_conv3x3_wgrad_tc", _p(x), xct, xco, _p(dy), dct, dco, n, H, W, ci, co, self._gw(name),
             _p(self.err), _sp())
        call("of_cnn_bias_grad", _p(dy), dct, dco, n * H * W, co, self._gb(name), _sp())

    def _relu_bwd(self, gt, gct, gco, yt, yct, yco, P, C):
        call("of_cnn_relu_bwd", _p(gt), gct, gco, _p(yt), yct, yco, P, C, _sp())

    def backward(self, b, g):
        """Gradients of the loss (dout from loss()) into self.grads (zeroed here)."""
        n, S = b["x0"].shape[0], b["x0"].shape[1]
        s1, s2, s3 = S // 2, S // 4, S // 8
        P0, P1, P2, P3 = n * S * S, n * s1 * s1, n * s2 * s2, n * s3 * s3
        self.grads.zero_()
        cv, wg, rb = self._conv, self._wgrad, self._relu_bwd
        # head (no ReLU)
        wg("head", b["d0"], 32, 0, g["dout"], 16, 0, n, S, S)
        cv("head", g["dout"], 16, 0, 16, n, S, S, g["d0"], 32, 0, flags=0, backward=True)
        rb(g["d0"], 32, 0, b["d0"], 32, 0, P0, 32)
        # dec0
        wg("d0", b["cat0"], 96, 0, g["d0"], 32, 0, n, S, S)
        cv("d0", g["d0"], 32, 0, 32, n, S, S, g["cat0"], 96, 0, flags=0, backward=True)
        call("of_cnn_upsample2_bwd", _p(g["cat0"]), 96, 0, n, s1, s1, 64, _p(g["d1"]), 64, 0, _sp())
        rb(g["d1"], 64, 0, b["d1"], 64, 0, P1, 64)
        # dec1
        wg("d1", b["cat1"], 192, 0, g["d1"], 64, 0, n, s1, s1)
        cv("d1", g["d1"], 64, 0, 64, n, s1, s1, g["cat1"], 192, 0, flags=0, backward=True)
        call("of_cnn_upsample2_bwd", _p(g["cat1"]), 192, 0, n, s2, s2, 128, _p(g["d2"]), 128, 0, _sp())
        rb(g["d2"], 128, 0, b["d2"], 128, 0, P2, 128)
        # dec2
        wg("d2", b["cat2"], 384, 0, g["d2"], 128, 0, n, s2, s2)
        cv("d2", g["d2"], 128, 0, 128, n, s2, s2, g["cat2"], 384, 0, flags=0, backward=True)
        call("of_cnn_upsample2_bwd", _p(g["cat2"]), 384, 0, n, s3, s3, 256, _p(g["e3"]), 256, 0, _sp())
        rb(g["e3"], 256, 0, b["e3"], 256, 0, P3, 256)
        # enc3
        wg("c3b", b["a3"], 256, 0, g["e3"], 256, 0, n, s3, s3)
        cv("c3b", g["e3"], 256, 0, 256, n, s3, s3, g["a3"], 256, 0, flags=0, backward=True)
        rb(g["a3"], 256, 0, b["a3"], 256, 0, P3, 256)
        wg("c3a", b["p3"], 128, 0, g["a3"], 256, 0, n, s3, s3)
        cv("c3a", g["a3"], 256, 0, 256, n, s3, s3, g["p3"], 128, 0, flags=0, backward=True)
        call("of_cnn_avgpool2_bwd", _p(g["p3"]), 128, 0, n, s2, s2, 128, _p(g["cat2"]), 384, 256, 1, _sp())
        rb(g["cat2"], 384, 256, b["cat2"], 384, 256, P2, 128)
        # enc2
        wg("c2b", b["a2"], 128, 0, g["cat2"], 384, 256, n, s2, s2)
        cv("c2b", g["cat2"], 384, 256, 128, n, s2, s2, g["a2"], 128, 0, flags=0, backward=True)
        rb(g["a2"], 128, 0, b["a2"], 128, 0, P2, 128)
        wg("c2a", b["p2"], 64, 0, g["a2"], 128, 0, n, s2, s2)
        cv("c2a", g["a2"], 128, 0, 128, n, s2, s2, g["p2"], 64, 0, flags=0, backward=True)
        call("of_cnn_avgpool2_bwd", _p(g["p2"]), 64, 0, n, s1, s1, 64, _p(g["cat1"]), 192, 128, 1, _sp())
        rb(g["cat1"], 192, 128, b["cat1"], 192, 128, P1, 64)
        # enc1
        wg("c1b", b["a1"], 64, 0, g["cat1"], 192, 128, n, s1, s1)
        cv("c1b", g["cat1"], 192, 128, 64, n, s1, s1, g["a1"], 64, 0, flags=0, backward=True)
        rb(g["a1"], 64, 0, b["a1"], 64, 0, P1, 64)
        wg("c1a", b["p1"], 32, 0, g["a1"], 64, 0, n, s1, s1)
        cv("c1a", g["a1"], 64, 0, 64, n, s1, s1, g["p1"], 32, 0, flags=0, backward=True)
        call("of_cnn_avgpool2_bwd", _p(g["p1"]), 32, 0, n, S, S, 32, _p(g["cat0"]), 96, 64, 1, _sp())
        rb(g["cat0"], 96, 64, b["cat0"], 96, 64, P0, 32)
        # enc0
        wg("c0b", b["a0"], 32, 0, g["cat0"], 96, 64, n, S, S)
        cv("c0b", g["cat0"], 96, 64, 32, n, S, S, g["a0"], 32, 0, flags=0, backward=True)
        rb(g["a0"], 32, 0, b["a0"], 32, 0, P0, 32)
        wg("c0a", b["x0"], IN_CH, 0, g["a0"], 32, 0, n, S, S)

    def check(self):
        """Raises if a convolution reported a timed-out wait since the last check."""
        e = int(self.err.item())
        if e:
            self.err.zero_()
            raise RuntimeError(f"of_cnn_conv3x3 reported error bits {e:#x}")


class LearnedLiuShen:
    """CNN warm start at the level 1/`factor` of the frame size, bilinear upsample, then at full size either
    Liu-Shen alone (mode "ls") or the pyramid's last level, Farneback (`fb_iters`
    iterations) then Liu-Shen (mode "fb"), with `sweeps` Liu-Shen sweeps.

    run() returns (U, V, iters, err): err is the solve's last update norm (device scalar);
    accept(err) tells whether it is within the calibrated threshold."""

    def __init__(self, net: WarmStartNet, sweeps=16, h=10.0, filter_opt=0.48, threshold=None, mode="ls", fb_iters=5,
                 factor=2):
        self.net, self.sweeps, self.h, self.filter_opt, self.threshold = net, int(sweeps), float(h), filter_opt, threshold
        if mode not in ("ls", "fb"):
            raise ValueError(mode)
        self.mode, self.fb_iters, self.factor = mode, int(fb_iters), int(factor)  # frame size / network size
        from gaussian_filter import prepareGaussianKernel
        self.taps = prepareGaussianKernel(filter_opt, 5)

    @classmethod
    def from_meta(cls, net, meta, start="cnn"):
        """The calibrated configuration.  The network was trained at meta["level"] for
        meta["frame"] (1024) frames; other frame sizes keep that ratio."""
        factor = int(meta.get("frame", 1024)) // int(meta.get("level", 512))
        if start == "cnn":
            return cls(net, sweeps=meta["sweeps"], threshold=meta["threshold"], mode=meta["mode"],
                       fb_iters=meta.get("fb_iters", 5), factor=factor)
        return cls(net, sweeps=meta.get("zero_sweeps", meta["sweeps"]), threshold=meta["threshold"], mode="fb",
                   fb_iters=meta.get("zero_fb_iters", 5), factor=factor)

    def pack(self, b, i, I0, I1):
        """The pyramid level the network runs at (1 / factor of the frames) of pair i into
        the network input (PIL bicubic, as the pyramid resizes)."""
        H, W = I0.shape
        n0 = ops.resize(I0, (W // self.factor, H // self.factor), bicubic=True)
        n1 = ops.resize(I1, (W // self.factor, H // self.factor), bicubic=True)
        self.net.pack_input(b, i, n0, n1)

    def upsample(self, out_i, H, W):
        """The network's (h, w, 2) flow -> the initial (U, V) at H x W: one fused bilinear
        kernel (the full-size stage refines it, so the pyramid's spline is not needed here)."""
        h, w, f = out_i.shape[0], out_i.shape[1], self.factor
        if (H, W) != (f * h, f * w):
            raise ValueError("frame and network sizes do not match the factor")
        U = torch.empty((H, W), dtype=torch.float32, device=out_i.device)
        V = torch.empty_like(U)
        call("of_cnn_flow_up", _p(out_i), h, w, f, _p(U), _p(V), W, float(f), _sp())
        return U, V

    def predict(self, I0, I1):
        """Initial (U, V) at the frames' size from the CNN at 1 / factor of it."""
        H, W = I0.shape
        b = self.net.buffers(1, H // self.factor)
        self.pack(b, 0, I0, I1)
        return self.upsample(self.net.forward(b)[0], H, W)

    def refine(self, I0, I1, U, V):
        """The full-size stage from the initial field: (Farneback,) then Liu-Shen.  U, V are
        handed over: the Farneback stage iterates on them in place."""
        if self.mode == "fb":
            import Farneback_PyCL as F
            U, V, _ = F.Farneback_PyCL(Niters=self.fb_iters)._compute_dev(I0, I1, U, V, consume_init=True)
        f0 = ops.prefilter(I0, self.taps)
        f1 = ops.prefilter(I1, self.taps)
        return ops.ls_solve(f0, f1, U, V, self.h, self.sweeps, 1e-8)

    def run(self, I0, I1):
        U, V = self.predict(I0, I1)
        return self.refine(I0, I1, U, V)

    def accept(self, err) -> bool:
        return self.threshold is None or float(err) <= self.threshold


def load_trained(path=WEIGHTS, device="cuda"):
    """The packaged network and its calibration (mode, sweeps, threshold, evaluation)."""
    import json
    d = np.load(path)
    meta = json.loads(str(d["meta"]))
    return WarmStartNet(device=device).load(path), meta


def _as_f32(t):
    """A float32 frame (uint8 / uint16 frames through the conversion kernel)."""
    return t if t.dtype == torch.float32 else ops.u8_to_f32(t)


class LearnedBatch:
    """n frame pairs of one size through the learned pipeline: one network forward over
    the batch, then each pair's full-size stage on one of `streams` CUDA streams; the
    whole step is captured into a CUDA graph on its first call and replayed afterwards.

    run() returns the per-pair (U, V) (graph-owned, overwritten by the next run) and a
    device vector of the Liu-Shen update norms; pairs whose norm exceeds the calibrated
    threshold are recomputed by the plain pyramid in fallback().

    start="zero" is the same full-size stage from a zero field with no network (the
    ablation the calibration compares against); it uses the calibration's zero-start
    Farneback iteration count."""

    def __init__(self, net, meta, n, size=1024, streams=4, use_graph=True, start="cnn"):
        if start not in ("cnn", "zero"):
            raise ValueError(start)
        self.ll = LearnedLiuShen.from_meta(net, meta, start)
        self.start = start
        self.net, self.n, self.size, self.nstreams, self.use_graph = net, int(n), int(size), max(1, streams), use_graph
        self._graph = None
        self._streams = None

    def _step(self, frames):
        cur = torch.cuda.current_stream()
        if self._streams is None:
            self._streams = [torch.cuda.Stream() for _ in range(self.nstreams)]
        # per pair, on its stream: uint8 / uint16 frames converted inside the graph, and the
        # network's input (the frames resized to its level) packed into the batch
        b = self.net.buffers(self.n, self.size // self.ll.factor) if self.start == "cnn" else None
        for s in self._streams:
            s.wait_stream(cur)
        conv = [None] * self.n
        for i, (A, B) in enumerate(frames):
            with torch.cuda.stream(self._streams[i % self.nstreams]):
                conv[i] = (_as_f32(A), _as_f32(B))
                if b is not None:
                    self.ll.pack(b, i, *conv[i])
        frames = conv
        out = None
        if b is not None:
            for s in self._streams:
                cur.wait_stream(s)
            out = self.net.forward(b)
            for s in self._streams:
                s.wait_stream(cur)
        errs = torch.empty(self.n, dtype=torch.float64, device=frames[0][0].device)
        res = [None] * self.n
        for i, (A, B) in enumerate(frames):
            with torch.cuda.stream(self._streams[i % self.nstreams]):
                if out is not None:
                    U, V = self.ll.upsample(out[i], self.size, self.size)
                else:
                    U, V = torch.zeros_like(A), torch.zeros_like(A)
                U, V, _, err = self.ll.refine(A, B, U, V)
                errs[i:i + 1].copy_(err.reshape(1))
                res[i] = (U, V)
        for s in self._streams:
            cur.wait_stream(s)
        return res, errs

    def run(self, frames):
        """frames: n (frame1, frame2) CUDA tensors of size x size (float32, uint8 or uint16)."""
        if len(frames) != self.n:
            raise ValueError("one frame pair per batch slot")
        if not self.use_graph:
            return self._step(frames)
        if self._graph is None:
            static_in = [(a.clone(), b.clone()) for a, b in frames]
            self._step(static_in)  # eager warm-up: sizes the buffers and workspaces
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.graph(g, stream=side):
                static_out = self._step(static_in)
            self._graph = (g, static_in, static_out)
        g, static_in, static_out = self._graph
        # all inputs into the graph's buffers with one multi-tensor copy
        torch._foreach_copy_([t for p in static_in for t in p], [t for p in frames for t in p])
        g.replay()
        return static_out

    def fallback(self, frames, res, errs):
        """Replaces the pairs whose update norm exceeds the threshold by the plain pyramid;
        returns the list of results and the number of pairs that fell back."""
        import Farneback_PyCL as F
        import GenericPyramidalOpticalFlow as G
        import PhysicsBasedOpticalFlowLiuShen as LS
        thr = self.ll.threshold
        if thr is None:
            return list(res), 0
        bad = (~(errs <= thr)).nonzero().flatten().tolist()  # NaN norms fall back too
        out = list(res)
        for i in bad:
            A, B = _as_f32(frames[i][0]), _as_f32(frames[i][1])
            out[i] = G.genericPyramidalOpticalFlow(A, B, 0, F.Farneback_PyCL(), 2, 1, 0.48,
                                                   LS.LiuShenOpticalFlowAlgoAdapter(10))
        return out, len(bad)
