"""The float32 Liu-Shen arithmetic (OF_LS_FAST, the library default).

It computes the reference's sweep in float32 with fused multiply-adds instead of the
reference's float64 stencil sums, so it is compared within tolerances:
  * against the bit-exact arithmetic on the same inputs: float32 rounding (<= 1e-4 px);
  * against the algorithm's float64 answer (oracle/oracle_f64.py) on the full-size
    Farneback pyr2 + Liu-Shen workload: <= 1e-3 px, endpoint error no worse (1e-5 px);
  * against the reference's own output at that size (every 8th pixel of its fields).
Every other property (borders, ragged shapes, the stop rule, batching) is checked too."""
import numpy as np
import pytest

import oracle_f64 as F
from conftest import golden

pytestmark = pytest.mark.gpu


def _frames(torch, size, seed=3):
    from gaussian_filter import prepareGaussianKernel
    from ofb200 import ops, synthetic as S
    a, b, _, _ = S.config_pair("fbls1024", seed=seed, size=size)
    taps = prepareGaussianKernel(0.48, 5)
    fa = ops.prefilter(torch.from_numpy(a.astype(np.float32)).cuda(), taps)
    fb = ops.prefilter(torch.from_numpy(b.astype(np.float32)).cuda(), taps)
    return fa, fb


def _solve(torch, fa, fb, arithmetic, tol=1e-8, maxnum=60, U0=None, V0=None):
    from ofb200 import ops
    U = torch.zeros_like(fa) if U0 is None else U0.clone()
    V = torch.zeros_like(fa) if V0 is None else V0.clone()
    U, V, it, e = ops.ls_solve(fa, fb, U, V, 10.0, maxnum, tol, arithmetic=arithmetic)
    return U.cpu().numpy(), V.cpu().numpy(), int(it.item()), float(e.item())


@pytest.mark.parametrize("shape", [(1024, 1024), (37, 300), (100, 57), (23, 56), (5, 9)])
def test_fast_matches_exact_to_float32_rounding(cuda_ok, shape):
    import torch
    g = torch.Generator().manual_seed(shape[0] * 7 + shape[1])
    fa = (torch.rand(shape, generator=g) * 200 + 20).cuda()
    fb = torch.roll(fa, shifts=(1, 1), dims=(0, 1)) + (torch.rand(shape, generator=g) * 4).cuda()
    U0 = (torch.randn(shape, generator=g) * 0.5).cuda()
    V0 = (torch.randn(shape, generator=g) * 0.5).cuda()
    ue, ve, ie, _ = _solve(torch, fa, fb, "exact", U0=U0, V0=V0)
    uf, vf, i_f, _ = _solve(torch, fa, fb, "fast", U0=U0, V0=V0)
    assert ie == i_f
    assert max(np.abs(ue - uf).max(), np.abs(ve - vf).max()) <= 1e-4
    assert not (np.array_equal(ue, uf) and np.array_equal(ve, vf)), "the float32 path should round differently"


def test_fast_piv_1024(cuda_ok):
    import torch
    fa, fb = _frames(torch, 1024)
    ue, ve, ie, ee = _solve(torch, fa, fb, "exact")
    uf, vf, i_f, ef = _solve(torch, fa, fb, "fast")
    assert ie == i_f == 60
    assert max(np.abs(ue - uf).max(), np.abs(ve - vf).max()) <= 1e-4
    assert ef == pytest.approx(ee, rel=1e-3)


@pytest.mark.parametrize("factor", [30.0, 3.0])
def test_fast_stop_rule(cuda_ok, factor):
    """With a tolerance the solve reaches before its 60th sweep (a multiple of the error
    left after 60 sweeps), both arithmetics stop early and within one sweep of each other."""
    import torch
    fa, fb = _frames(torch, 256, seed=5)
    _, _, n60, e60 = _solve(torch, fa, fb, "exact", tol=0.0)
    assert n60 == 60
    _, _, ie, _ = _solve(torch, fa, fb, "exact", tol=factor * e60)
    _, _, i_f, _ = _solve(torch, fa, fb, "fast", tol=factor * e60)
    assert ie < 60 and abs(ie - i_f) <= 1


def test_fast_pipeline_against_float64_and_reference(cuda_ok):
    """LiuSE_Farneback_Fs0_0_PyrLvls2 at 1024^2 with the float32 sweep."""
    import Farneback_PyCL as FB
    import GenericPyramidalOpticalFlow as G
    import PhysicsBasedOpticalFlowLiuShen as LS
    from ofb200 import synthetic as S
    a8, b8, Ug, Vg = S.config_pair("fbls1024", seed=1)
    a, b = a8.astype(np.float32), b8.astype(np.float32)
    U, V = G.genericPyramidalOpticalFlow(a.copy(), b.copy(), 0, FB.Farneback_PyCL(), 2, 1, 0.48,
                                         LS.LiuShenOpticalFlowAlgoAdapter(10, arithmetic="fast"))
    U6, V6 = F.pyramid(a, b, 0, F.FB(), 2, 1, 0.48, F.LS(10))
    assert max(np.abs(U - U6).max(), np.abs(V - V6).max()) <= 1e-3
    e32 = S.epe(U, V, Ug, Vg, crop=16)
    e64 = S.epe(U6.astype(np.float32), V6.astype(np.float32), Ug, Vg, crop=16)
    assert e32 <= e64 + 1e-5
    g = golden("configs")
    assert max(np.abs(U[::8, ::8] - g["fbls1024_Uref8"]).max(), np.abs(V[::8, ::8] - g["fbls1024_Vref8"]).max()) <= 1e-3


def test_fast_batch_equals_single_pairs(cuda_ok):
    """PairBatch (several streams, one CUDA graph) gives the single-pair results exactly."""
    import torch
    import Farneback_PyCL as FB
    import GenericPyramidalOpticalFlow as G
    import PhysicsBasedOpticalFlowLiuShen as LS
    from ofb200 import ops, synthetic as S
    from ofb200.batch import PairBatch, PairSpec
    frames = []
    for s in range(3):
        a, b, _, _ = S.config_pair("fbls1024", seed=30 + s, size=256)
        frames.append((torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()))
    spec = PairSpec(0, lambda: FB.Farneback_PyCL(), 2, 1, 0.48,
                    lambda: LS.LiuShenOpticalFlowAlgoAdapter(10, arithmetic="fast"), key=("fbls-fast",))
    out = PairBatch([spec] * 3, streams=3).run(frames)
    for (a8, b8), (U, V) in zip(frames, out):
        Us, Vs = G.genericPyramidalOpticalFlow(ops.u8_to_f32(a8), ops.u8_to_f32(b8), 0, FB.Farneback_PyCL(), 2, 1, 0.48,
                                               LS.LiuShenOpticalFlowAlgoAdapter(10, arithmetic="fast"))
        assert torch.equal(U, Us) and torch.equal(V, Vs)
