"""The learned warm start's kernels against the CPU oracle (oracle/cnn_oracle.py).

Convolutions accumulate in float32 on the tensor cores and round the output to bfloat16,
so they are compared with a tolerance of one bfloat16 step (2^-7 relative) plus 1e-5 of
the output's scale; the elementwise kernels and Adam are bit-exact; network gradients are
compared per layer by relative L2 error (< 5e-2) and cosine similarity (> 0.998)."""
import ctypes
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _P(t):
    return ctypes.c_void_p(t.data_ptr())


def _sp():
    from ofb200 import ops
    return ops.stream_ptr()


def _bf(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda().to(torch.bfloat16)


def _f(t):
    return t.float().cpu().numpy()


def _conv(torch, x, cin, xco, w9, bias, flags, cout_store=None, y_ctot=None, y_coff=0, f32=False):
    from ofb200._lib import call
    n, H, W, xct = x.shape
    cout = w9.shape[1]
    wb = _bf(torch, w9)
    y_ctot = y_ctot or cout
    y = torch.zeros((n, H, W, y_ctot), dtype=torch.float32 if f32 else torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    b = None if bias is None else torch.from_numpy(bias.astype(np.float32)).cuda()
    call("of_cnn_conv3x3", _P(x), n, H, W, cin, xct, xco, _P(wb), cout, None if b is None else _P(b), flags, _P(y),
         y_ctot, y_coff, cout_store or cout, _P(err), _sp())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return y


def _close(got, want, rtol=2.0 ** -7):
    scale = max(float(np.max(np.abs(want))), 1e-30)
    bad = np.abs(got - want) > rtol * np.abs(want) + 1e-5 * scale
    assert not bad.any(), (int(bad.sum()), float(np.max(np.abs(got - want))), scale)


CONV_CASES = [  # n, H, W, cin, cout, relu
    (2, 32, 32, 16, 32, True),
    (1, 64, 64, 32, 64, True),
    (1, 16, 16, 64, 128, False),
    (1, 32, 64, 96, 32, True),
    (1, 16, 16, 256, 256, True),
    (1, 32, 32, 384, 384, False),
    (1, 8, 256, 128, 16, False),
    (3, 16, 32, 192, 64, True),
    (4, 8, 8, 256, 256, True),
    (2, 8, 16, 128, 64, False),
    # rows of 128 pixels: the 9 taps as views of one 3 x 130 halo box
    (2, 16, 128, 16, 32, True),
    (1, 8, 128, 32, 32, False),
    (1, 6, 128, 64, 64, True),
    (1, 4, 256, 96, 32, True),
    (1, 4, 128, 384, 384, False),
    (1, 4, 128, 256, 256, True),
    (2, 3, 128, 192, 64, True),
]


@pytest.mark.parametrize("case", CONV_CASES, ids=[str(c) for c in CONV_CASES])
def test_conv_forward(torch_cuda, case):
    import cnn_oracle as C
    torch = torch_cuda
    n, H, W, cin, cout, relu = case
    rng = np.random.default_rng(hash(case) % 2 ** 32)
    x = C.bf16(rng.normal(0, 1, (n, H, W, cin)))
    w = C.bf16(rng.normal(0, 1.0 / np.sqrt(9 * cin), (9, cout, cin)))
    b = rng.normal(0, 0.1, cout).astype(np.float32)
    y = _conv(torch, _bf(torch, x), cin, 0, w, b, 1 if relu else 0)
    want = C.conv3x3(x, w, b)
    if relu:
        want = np.maximum(want, 0)
    _close(_f(y), want)


def test_conv_channel_slices_and_f32_head(torch_cuda):
    """Input read from, and output written into, channel slices of wider tensors; the
    head's float32 store of the first 2 of 16 channels."""
    import cnn_oracle as C
    torch = torch_cuda
    rng = np.random.default_rng(5)
    full = C.bf16(rng.normal(0, 1, (2, 32, 32, 96)))
    w = C.bf16(rng.normal(0, 0.1, (9, 32, 32)))
    y = _conv(torch, _bf(torch, full), 32, 64, w, None, 1, y_ctot=96, y_coff=32)
    want = np.maximum(C.conv3x3(full[..., 64:], w), 0)
    got = _f(y)
    _close(got[..., 32:64], want)
    assert not got[..., :32].any() and not got[..., 64:].any()
    wh = np.zeros((9, 16, 32), np.float32)
    wh[:, :2] = C.bf16(rng.normal(0, 0.1, (9, 2, 32)))
    bh = np.zeros(16, np.float32)
    bh[:2] = [0.5, -0.25]
    y2 = _conv(torch, _bf(torch, full[..., :32].copy()), 32, 0, wh, bh, 2, cout_store=2, y_ctot=2, f32=True)
    _close(y2.cpu().numpy(), C.conv3x3(full[..., :32], wh[:, :2], bh[:2]))


def test_conv_input_gradient_via_packed_weights(torch_cuda):
    import cnn_oracle as C
    from ofb200._lib import call
    torch = torch_cuda
    rng = np.random.default_rng(6)
    cin, cout = 96, 32
    w = rng.normal(0, 0.1, (9, cout, cin)).astype(np.float32)
    wt = torch.from_numpy(w).cuda()
    wb = torch.empty((9, cin, cout), dtype=torch.bfloat16, device="cuda")
    call("of_cnn_pack_weights", _P(wt), cout, cin, cout, cin, 1, _P(wb), _sp())
    wf = torch.empty((9, cout, cin), dtype=torch.bfloat16, device="cuda")
    call("of_cnn_pack_weights", _P(wt), cout, cin, cout, cin, 0, _P(wf), _sp())
    torch.cuda.synchronize()
    assert np.array_equal(_f(wf), C.bf16(w))
    wbn = _f(wb)
    for t in range(9):
        assert np.array_equal(wbn[t], C.bf16(w[8 - t]).T)
    dy = C.bf16(rng.normal(0, 1, (1, 32, 32, cout)))
    y = _conv(torch, _bf(torch, dy), cout, 0, wbn, None, 0)
    _close(_f(y), C.conv3x3_dgrad(dy, C.bf16(w)))


@pytest.mark.parametrize("cin,cout,coff", [(2, 32, 0), (32, 64, 64), (96, 32, 0), (256, 256, 0), (32, 2, 0)])
def test_weight_gradient(torch_cuda, cin, cout, coff):
    import cnn_oracle as C
    from ofb200._lib import call
    torch = torch_cuda
    rng = np.random.default_rng(cin * 1000 + cout)
    n, H, W = 2, 16, 80
    xct = max(16, cin + coff)
    x = C.bf16(rng.normal(0, 1, (n, H, W, xct)))
    dct = max(16, cout)
    dy = C.bf16(rng.normal(0, 1, (n, H, W, dct)))
    dw = torch.zeros((9, cout, cin), dtype=torch.float32, device="cuda")
    db = torch.zeros(cout, dtype=torch.float32, device="cuda")
    xt, dyt = _bf(torch, x), _bf(torch, dy)
    call("of_cnn_conv3x3_wgrad", _P(xt), xct, coff, _P(dyt), dct, 0, n, H, W, cin, cout, _P(dw), _sp())
    call("of_cnn_bias_grad", _P(dyt), dct, 0, n * H * W, cout, _P(db), _sp())
    torch.cuda.synchronize()
    want = C.conv3x3_wgrad(x[..., coff:coff + cin], dy[..., :cout])
    got = dw.cpu().numpy()
    assert np.max(np.abs(got - want)) <= 1e-4 * np.max(np.abs(want))
    wb = dy[..., :cout].astype(np.float64).sum(axis=(0, 1, 2))
    assert np.max(np.abs(db.cpu().numpy() - wb)) <= 1e-4 * np.max(np.abs(wb))


def test_pool_and_upsample_any_channel_layout(torch_cuda):
    """Channel counts and offsets that are not multiples of 8 take the one-channel-per-thread
    kernels; multiples of 8 the 8-channel ones: both equal the oracle."""
    import cnn_oracle as C
    from ofb200._lib import call
    torch = torch_cuda
    rng = np.random.default_rng(9)
    n, H, W = 3, 10, 14
    x = C.bf16(rng.normal(0, 1, (n, H, W, 24)))
    xt = _bf(torch, x)
    for c0, cn in ((4, 12), (2, 5), (8, 8), (0, 16)):
        p = torch.empty((n, H // 2, W // 2, cn), dtype=torch.bfloat16, device="cuda")
        call("of_cnn_avgpool2", _P(xt), 24, c0, n, H, W, cn, _P(p), cn, 0, _sp())
        up = torch.zeros((n, 2 * H, 2 * W, cn), dtype=torch.bfloat16, device="cuda")
        call("of_cnn_upsample2", _P(xt), 24, c0, n, H, W, cn, _P(up), cn, 0, _sp())
        torch.cuda.synchronize()
        assert np.array_equal(_f(p), C.bf16(C.avgpool2(x[..., c0:c0 + cn]))), (c0, cn)
        assert np.array_equal(_f(up), C.upsample2(x[..., c0:c0 + cn])), (c0, cn)


def test_elementwise_kernels_bit_exact(torch_cuda):
    import cnn_oracle as C
    from ofb200._lib import call
    torch = torch_cuda
    rng = np.random.default_rng(7)
    n, H, W = 2, 16, 24
    x = C.bf16(rng.normal(0, 1, (n, H, W, 48)))
    xt = _bf(torch, x)
    p = torch.empty((n, H // 2, W // 2, 32), dtype=torch.bfloat16, device="cuda")
    call("of_cnn_avgpool2", _P(xt), 48, 16, n, H, W, 32, _P(p), 32, 0, _sp())
    torch.cuda.synchronize()
    assert np.array_equal(_f(p), C.bf16(C.avgpool2(x[..., 16:])))
    acc = C.bf16(rng.normal(0, 1, (n, H, W, 48)))
    acct = _bf(torch, acc)
    call("of_cnn_avgpool2_bwd", _P(p), 32, 0, n, H, W, 32, _P(acct), 48, 8, 1, _sp())
    torch.cuda.synchronize()
    want = acc.copy()
    want[..., 8:40] = C.bf16(C.avgpool2_bwd(_f(p)) + acc[..., 8:40])
    assert np.array_equal(_f(acct), want)
    up = torch.zeros((n, 2 * H, 2 * W, 64), dtype=torch.bfloat16, device="cuda")
    call("of_cnn_upsample2", _P(xt), 48, 0, n, H, W, 32, _P(up), 64, 32, _sp())
    torch.cuda.synchronize()
    assert np.array_equal(_f(up)[..., 32:], C.upsample2(x[..., :32]))
    g = C.bf16(rng.normal(0, 1, (n, 2 * H, 2 * W, 64)))
    gt = _bf(torch, g)
    d = torch.empty((n, H, W, 32), dtype=torch.bfloat16, device="cuda")
    call("of_cnn_upsample2_bwd", _P(gt), 64, 32, n, H, W, 32, _P(d), 32, 0, _sp())
    torch.cuda.synchronize()
    assert np.array_equal(_f(d), C.bf16(C.upsample2_bwd(g[..., 32:])))
    call("of_cnn_relu_bwd", _P(gt), 64, 0, _P(up), 64, 0, n * 4 * H * W, 64, _sp())
    torch.cuda.synchronize()
    assert np.array_equal(_f(gt), np.where(_f(up) > 0, g, 0))


@pytest.mark.parametrize("H,W", [(24, 40), (300, 260)])
def test_pack_pair_and_split_flow(torch_cuda, H, W):
    """The network input: one CTA for small frames, the multi-block maxima above 64 K pixels."""
    import cnn_oracle as C
    from ofb200._lib import call
    torch = torch_cuda
    rng = np.random.default_rng(8)
    a = rng.uniform(0, 200, (H, W)).astype(np.float32)
    b = rng.uniform(0, 250, (H, W)).astype(np.float32)
    at, bt = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    mx = torch.full((2,), 7, dtype=torch.int32, device="cuda")  # stale contents are overwritten
    out = torch.empty((H, W, 16), dtype=torch.bfloat16, device="cuda")
    call("of_cnn_pack_pair", _P(at), _P(bt), H, W, W, _P(mx), _P(out), 16, _sp())
    torch.cuda.synchronize()
    o = _f(out)
    assert np.array_equal(o[..., 0], C.bf16(a / a.max())) and np.array_equal(o[..., 1], C.bf16(b / b.max()))
    assert not o[..., 2:].any()
    assert mx.cpu().numpy().view(np.float32).tolist() == [a.max(), b.max()]
    if (H, W) != (24, 40):
        return
    f = rng.normal(0, 1, (24, 40, 2)).astype(np.float32)
    ft = torch.from_numpy(f).cuda()
    u = torch.empty((24, 48), dtype=torch.float32, device="cuda")[:, :40]
    v = torch.empty((24, 48), dtype=torch.float32, device="cuda")[:, :40]
    call("of_cnn_split_flow", _P(ft), 24, 40, _P(u), _P(v), 48, _sp())
    torch.cuda.synchronize()
    assert np.array_equal(u.cpu().numpy(), f[..., 0]) and np.array_equal(v.cpu().numpy(), f[..., 1])


def test_loss_and_adam_bit_exact(torch_cuda):
    import cnn_oracle as C
    from ofb200._lib import call
    torch = torch_cuda
    rng = np.random.default_rng(9)
    pred = rng.normal(0, 1, (2, 8, 8, 2)).astype(np.float32)
    lab = rng.normal(0, 1, (2, 8, 8, 2)).astype(np.float32)
    pt, lt = torch.from_numpy(pred).cuda(), torch.from_numpy(lab).cuda()
    g = torch.empty((2, 8, 8, 16), dtype=torch.bfloat16, device="cuda")
    loss = torch.zeros((), dtype=torch.float64, device="cuda")
    call("of_cnn_flow_mse", _P(pt), _P(lt), 128, _P(g), 16, _P(loss), _sp())
    torch.cuda.synchronize()
    lw, dw = C.flow_mse(pred, lab)
    assert abs(float(loss.item()) - lw) <= 1e-6 * lw
    assert np.array_equal(_f(g)[..., :2], C.bf16(dw)) and not _f(g)[..., 2:].any()
    w = rng.normal(0, 1, 1000).astype(np.float32)
    gr = rng.normal(0, 1e-3, 1000).astype(np.float32)
    m = np.zeros(1000, np.float32)
    v = np.zeros(1000, np.float32)
    wt, gt, mt, vt = (torch.from_numpy(a.copy()).cuda() for a in (w, gr, m, v))
    for step in (1, 2, 3):
        call("of_cnn_adam", _P(wt), _P(gt), _P(mt), _P(vt), 1000, 1e-3, 0.9, 0.999, 1e-8, step, _sp())
        w, m, v = C.adam(w, gr, m, v, step, 1e-3)
    torch.cuda.synchronize()
    assert np.array_equal(wt.cpu().numpy(), w) and np.array_equal(mt.cpu().numpy(), m)
    assert np.array_equal(vt.cpu().numpy(), v)


def _relerr(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _cos(a, b):
    return float(np.dot(a.ravel(), b.ravel()) / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30))


def test_network_gradients_match_oracle(torch_cuda):
    """Forward and backward of the whole network (n = 2, 64 x 64) against the oracle."""
    import cnn_oracle as C
    torch = torch_cuda
    from ofb200.warmstart import LAYERS, WarmStartNet
    net = WarmStartNet(seed=4)
    rng = np.random.default_rng(10)
    x = C.bf16(rng.uniform(0, 1, (2, 64, 64, 2)))
    lab = rng.normal(0, 1, (2, 64, 64, 2)).astype(np.float32)
    b = net.buffers(2, 64)
    gb = net.grad_buffers(2, 64)
    b["x0"].zero_()
    b["x0"][..., :2] = _bf(torch, x)
    labt = torch.from_numpy(lab).cuda()
    out = net.forward(b)
    loss = net.loss(b, gb, labt)
    net.backward(b, gb)
    torch.cuda.synchronize()
    net.check()
    on = C.Net(C.flat_to_params(net.params.cpu().numpy()))
    oo = on.forward(x)
    assert _relerr(out.cpu().numpy(), oo) < 1e-2
    lw, dw = C.flow_mse(oo, lab)
    assert abs(float(loss.item()) - lw) < 1e-2 * lw
    og = on.backward(dw)
    gflat = net.grads.cpu().numpy()
    for name, ci, co in LAYERS:
        wo, bo, _, _ = net.off[name]
        gw = gflat[wo:bo].reshape(9, co, ci)
        gbias = gflat[bo:bo + co]
        assert _relerr(gw, og[name][0]) < 5e-2, name
        assert _cos(gw, og[name][0]) > 0.998, name
        assert _relerr(gbias, og[name][1]) < 5e-2, name


def test_training_reduces_loss(torch_cuda):
    torch = torch_cuda
    from ofb200.warmstart import WarmStartNet
    net = WarmStartNet(seed=1)
    rng = np.random.default_rng(11)
    b = net.buffers(4, 64)
    gb = net.grad_buffers(4, 64)
    b["x0"].zero_()
    b["x0"][..., :2] = torch.from_numpy(rng.uniform(0, 1, (4, 64, 64, 2)).astype(np.float32)).cuda().to(torch.bfloat16)
    yy, xx = np.mgrid[0:64, 0:64] / 64.0
    lab = np.stack([np.sin(2 * np.pi * yy), np.cos(2 * np.pi * xx)], -1)[None].repeat(4, 0).astype(np.float32)
    labt = torch.from_numpy(lab).cuda()
    losses = []
    for _ in range(120):
        net.forward(b)
        losses.append(float(net.loss(b, gb, labt).item()))
        net.backward(b, gb)
        net.adam(1e-3)
    net.check()
    # the weight gradients are summed with atomics, so the trajectory varies between runs
    assert min(losses[-20:]) < 0.3 * losses[0], losses[::10]


WGRAD_TC_CASES = [  # n, H, W, cin, cout, x channel offset
    (2, 16, 64, 2, 32, 0), (2, 16, 64, 32, 64, 64), (2, 16, 64, 96, 32, 0), (1, 8, 128, 256, 256, 0),
    (2, 16, 64, 32, 2, 0), (1, 8, 64, 384, 128, 0), (2, 8, 64, 192, 64, 0), (4, 8, 8, 128, 128, 0),
    (2, 4, 8, 64, 32, 0), (1, 64, 64, 32, 32, 0),
]


@pytest.mark.parametrize("case", WGRAD_TC_CASES, ids=[str(c) for c in WGRAD_TC_CASES])
def test_weight_gradient_tensor_cores(torch_cuda, case):
    """The tcgen05 weight gradient against the oracle (f32 accumulation in another order)."""
    import cnn_oracle as C
    from ofb200._lib import call
    torch = torch_cuda
    n, H, W, cin, cout, coff = case
    rng = np.random.default_rng(cin * 7 + cout + H)
    xct = max(16, (cin + coff + 7) // 8 * 8)
    dct = max(16, (cout + 7) // 8 * 8)
    x = C.bf16(rng.normal(0, 1, (n, H, W, xct)))
    dy = C.bf16(rng.normal(0, 1, (n, H, W, dct)))
    dw = torch.zeros((9, cout, cin), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    xt, dyt = _bf(torch, x), _bf(torch, dy)
    call("of_cnn_conv3x3_wgrad_tc", _P(xt), xct, coff, _P(dyt), dct, 0, n, H, W, cin, cout, _P(dw), _P(err), _sp())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    want = C.conv3x3_wgrad(x[..., coff:coff + cin], dy[..., :cout])
    got = dw.cpu().numpy()
    assert np.max(np.abs(got - want)) <= 1e-4 * np.max(np.abs(want)), float(np.max(np.abs(got - want)))


@pytest.mark.parametrize("factor", [2, 4])
def test_flow_upsample_bilinear(torch_cuda, factor):
    """The learned start's fused upsample against a float64 restatement (pixel-centre
    bilinear, clamped edges, displacements times the factor)."""
    from ofb200._lib import call
    torch = torch_cuda
    rng = np.random.default_rng(13)
    h, w, f = 12, 20, factor
    fl = rng.normal(0, 1, (h, w, 2)).astype(np.float32)
    ft = torch.from_numpy(fl).cuda()
    U = torch.empty((f * h, f * w), dtype=torch.float32, device="cuda")
    V = torch.empty_like(U)
    call("of_cnn_flow_up", _P(ft), h, w, f, _P(U), _P(V), f * w, float(f), _sp())
    torch.cuda.synchronize()
    sy = np.maximum((np.arange(f * h) + 0.5) / f - 0.5, 0)
    sx = np.maximum((np.arange(f * w) + 0.5) / f - 0.5, 0)
    y0 = np.minimum(np.floor(sy).astype(int), h - 1)
    x0 = np.minimum(np.floor(sx).astype(int), w - 1)
    y1, x1 = np.minimum(y0 + 1, h - 1), np.minimum(x0 + 1, w - 1)
    ay, ax = (sy - y0)[:, None], (sx - x0)[None, :]
    for c, got in ((0, U), (1, V)):
        g = fl[..., c].astype(np.float64)
        top = g[y0][:, x0] + ax * (g[y0][:, x1] - g[y0][:, x0])
        bot = g[y1][:, x0] + ax * (g[y1][:, x1] - g[y1][:, x0])
        want = f * (top + ay * (bot - top))
        assert np.max(np.abs(got.cpu().numpy() - want)) <= 1e-5 * f
