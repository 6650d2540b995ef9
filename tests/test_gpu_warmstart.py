"""The learned Liu-Shen warm start end to end: the batched, graph-replayed pipeline equals
the single-pair one (1024^2 frames), and on held-out pairs of the 1024^2 workload (seeds outside both the
training and the calibration sets) the packaged network gives a lower interior endpoint
error than the plain pyramid and than the same full-size stage started from zero."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HELD_OUT = (950_000, 950_001)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def trained(torch_cuda):
    from ofb200.warmstart import load_trained
    return load_trained()


def _f32(torch, a):
    return torch.from_numpy(a.astype(np.float32)).cuda()


def test_batch_matches_single_pair(torch_cuda, trained):
    torch = torch_cuda
    from ofb200 import synthetic as S
    from ofb200.warmstart import LearnedBatch, LearnedLiuShen
    net, meta = trained
    frames = []
    for seed in (1, 2, 3):  # the benchmark's frame size: the network's deepest scale fills its tiles
        a, b, _, _ = S.config_pair("fbls1024", seed=seed)
        frames.append((_f32(torch, a), _f32(torch, b)))
    ll = LearnedLiuShen.from_meta(net, meta)
    want = [ll.run(A, B) for A, B in frames]
    want = [(U.cpu().numpy(), V.cpu().numpy(), float(e.item())) for U, V, _, e in want]
    lb = LearnedBatch(net, meta, 3, size=1024, streams=2)
    for _ in range(2):  # capture, then replay
        res, errs = lb.run(frames)
        torch.cuda.synchronize()
        for (U, V), e, (Uw, Vw, ew) in zip(res, errs.cpu().tolist(), want):
            assert np.array_equal(U.cpu().numpy(), Uw) and np.array_equal(V.cpu().numpy(), Vw)
            assert e == pytest.approx(ew, rel=1e-9)  # summed with float64 atomics in any order
    net.check()


def test_trained_start_gain(torch_cuda, trained):
    """With the calibrated configuration (one Farneback iteration at full size, then a few
    Liu-Shen sweeps) the network's start is at least as accurate as the plain pyramid and
    far better than the same stage from zero, which needs a second Farneback iteration to
    come close: that iteration is what the network saves."""
    torch = torch_cuda
    import Farneback_PyCL as F
    import GenericPyramidalOpticalFlow as G
    import PhysicsBasedOpticalFlowLiuShen as LS
    from ofb200 import synthetic as S
    from ofb200.warmstart import LearnedLiuShen
    net, meta = trained
    assert meta["mode"] == "fb" and meta["fb_iters"] < meta["zero_fb_iters"]
    ll = LearnedLiuShen.from_meta(net, meta)
    e_plain, e_learned, e_zero = [], [], []
    for seed in HELD_OUT:
        a, b, Ug, Vg = S.config_pair("fbls1024", seed=seed)
        A, B = _f32(torch, a), _f32(torch, b)
        Up, Vp = G.genericPyramidalOpticalFlow(A, B, 0, F.Farneback_PyCL(), 2, 1, 0.48,
                                               LS.LiuShenOpticalFlowAlgoAdapter(10))
        e_plain.append(S.epe(Up.cpu().numpy(), Vp.cpu().numpy(), Ug, Vg, crop=16))
        U, V, _, err = ll.run(A, B)
        e_learned.append(S.epe(U.cpu().numpy(), V.cpu().numpy(), Ug, Vg, crop=16))
        assert float(err.item()) <= meta["threshold"]  # within the calibrated acceptance threshold
        Z = torch.zeros_like(A)
        Uz, Vz, _, _ = ll.refine(A, B, Z, Z.clone())
        e_zero.append(S.epe(Uz.cpu().numpy(), Vz.cpu().numpy(), Ug, Vg, crop=16))
    net.check()
    assert np.mean(e_learned) <= np.mean(e_plain), (e_learned, e_plain)
    assert np.mean(e_learned) < 0.5 * np.mean(e_zero), (e_learned, e_zero)


def test_fallback_returns_the_plain_pyramid(torch_cuda, trained):
    """A pair the network cannot start well (two unrelated frames: no displacement explains
    the second) ends its reduced Liu-Shen stage with an update norm above the calibrated
    threshold; fallback() then recomputes it with the plain pyramid, whose result is what
    comes back, while an ordinary pair of the same batch keeps its learned result."""
    torch = torch_cuda
    import Farneback_PyCL as F
    import GenericPyramidalOpticalFlow as G
    import PhysicsBasedOpticalFlowLiuShen as LS
    from ofb200 import synthetic as S
    from ofb200.warmstart import LearnedBatch
    net, meta = trained
    a, b, _, _ = S.config_pair("fbls1024", seed=HELD_OUT[0])
    c, _, _, _ = S.config_pair("fbls1024", seed=HELD_OUT[1] + 77)
    frames = [(_f32(torch, a), _f32(torch, b)), (_f32(torch, a), _f32(torch, c))]
    lb = LearnedBatch(net, meta, 2, size=1024, streams=2)
    res, errs = lb.run(frames)
    e = errs.cpu().tolist()
    assert e[0] <= meta["threshold"] and not e[1] <= meta["threshold"], e
    learned0 = (res[0][0].clone(), res[0][1].clone())
    out, nfb = lb.fallback(frames, res, errs.cpu())
    assert nfb == 1
    Up, Vp = G.genericPyramidalOpticalFlow(frames[1][0], frames[1][1], 0, F.Farneback_PyCL(), 2, 1, 0.48,
                                           LS.LiuShenOpticalFlowAlgoAdapter(10))
    assert torch.equal(out[1][0], Up) and torch.equal(out[1][1], Vp)
    assert torch.equal(out[0][0], learned0[0]) and torch.equal(out[0][1], learned0[1])


def test_large_displacement_network(torch_cuda):
    """The network trained on 2-16 px flows (warmstart_weights_12px.npz), on held-out pairs
    with displacements up to 12 px: with its calibrated stage (one Farneback iteration and
    a few Liu-Shen sweeps) it is at least as accurate as the plain pyramid, while the same
    stage from a zero start, with the calibration's most expensive zero-start stage, is far
    off: at these displacements the start needs the coarse level, and the network gives it."""
    torch = torch_cuda
    import os
    import Farneback_PyCL as F
    import GenericPyramidalOpticalFlow as G
    import PhysicsBasedOpticalFlowLiuShen as LS
    from ofb200 import synthetic as S
    from ofb200.warmstart import WEIGHTS, LearnedLiuShen, load_trained
    net, meta = load_trained(path=os.path.join(os.path.dirname(WEIGHTS), "warmstart_weights_12px.npz"))
    assert meta["eval_max_disp"] == 12.0
    ll = LearnedLiuShen.from_meta(net, meta)
    llz = LearnedLiuShen.from_meta(net, meta, "zero")
    e_plain, e_learned, e_zero = [], [], []
    for seed in (975_000, 975_001):
        a, b, Ug, Vg = S.piv_pair(1024, 1024, "fourier", seed, density=0.05, diameter=(2.0, 3.0), noise=2.0,
                                  max_disp=12.0)
        A, B = _f32(torch, a), _f32(torch, b)
        Up, Vp = G.genericPyramidalOpticalFlow(A, B, 0, F.Farneback_PyCL(), 2, 1, 0.48,
                                               LS.LiuShenOpticalFlowAlgoAdapter(10))
        e_plain.append(S.epe(Up.cpu().numpy(), Vp.cpu().numpy(), Ug, Vg, crop=16))
        U, V, _, err = ll.run(A, B)
        e_learned.append(S.epe(U.cpu().numpy(), V.cpu().numpy(), Ug, Vg, crop=16))
        Z = torch.zeros_like(A)
        Uz, Vz, _, _ = llz.refine(A, B, Z, Z.clone())
        e_zero.append(S.epe(Uz.cpu().numpy(), Vz.cpu().numpy(), Ug, Vg, crop=16))
    net.check()
    assert np.mean(e_learned) <= np.mean(e_plain), (e_learned, e_plain)
    assert np.mean(e_zero) > 3 * np.mean(e_plain), (e_zero, e_plain)
