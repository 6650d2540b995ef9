"""GPU parity: every kernel of the hot path against the reference's own outputs (golden
fixtures from tests/golden/make_golden.py) and against the CPU oracle.

Bar: bit-exact (np.array_equal) wherever the oracle is bit-exact with the reference;
flow fields of full pipelines within 1e-3 px max-abs; the spline upsample within 1 float32
ulp of scipy.
"""
import numpy as np
import pytest

import oracle as O
from conftest import golden

pytestmark = pytest.mark.gpu

TOL_PX = 1e-3  # max-abs flow tolerance of the parity contract


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def rng(seed=0):
    return np.random.default_rng(seed)


# ------------------------------------------------------------------------------ A1
def test_prefilter_golden(torch_cuda):
    from ofb200 import ops
    g = golden("prefilter")
    for i, (s, K) in enumerate([(3.4, 3), (2.0, 3), (0.48, 5)]):
        out = ops.prefilter(dev(torch_cuda, g["img"]), O.prepare_gaussian_kernel(s, K))
        assert np.array_equal(host(out), g[f"out{i}"])


@pytest.mark.parametrize("shape", [(1, 7), (5, 3), (64, 64), (129, 257), (1024, 1024)])
@pytest.mark.parametrize("K,s", [(3, 3.4), (5, 0.48), (9, 1.2), (15, 2.5), (73, 0.6 * 3)])
def test_prefilter_vs_oracle(torch_cuda, shape, K, s):
    from ofb200 import ops
    img = rng(1).uniform(0, 255, shape).astype(np.float32)
    if min(shape) < K // 2:  # the reference raises IndexError here, and so does the drop-in
        import gaussian_filter as GF
        with pytest.raises(IndexError):
            GF.gaussian_filterPx(img.copy(), s, K)
        return
    taps = O.prepare_gaussian_kernel(s, K)
    out = ops.prefilter(dev(torch_cuda, img), taps)
    assert np.array_equal(host(out), O.prefilter_taps(img, taps))
    u8 = np.round(img).astype(np.uint8)
    out8 = ops.prefilter(dev(torch_cuda, u8), taps)
    assert np.array_equal(host(out8), O.prefilter_taps(u8.astype(np.float32), taps))


def test_prefilter_pitched_planes(torch_cuda):
    from ofb200 import ops
    img = rng(2).uniform(0, 255, (40, 50)).astype(np.float32)
    big = torch_cuda.zeros((40, 64), device="cuda")
    big[:, :50] = dev(torch_cuda, img)
    out = ops.prefilter(big[:, :50], O.prepare_gaussian_kernel(3.4, 3))
    assert np.array_equal(host(out), O.prefilter(img, 3.4, 3))


# ------------------------------------------------------------------------------ A2/A3/A4
def test_resize_golden(torch_cuda):
    from ofb200 import ops
    g = golden("resize")
    i = 0
    while f"src{i}" in g:
        W, H, f = g[f"spec{i}"]
        out = ops.resize(dev(torch_cuda, g[f"src{i}"]), (int(W), int(H)), bool(f))
        assert np.array_equal(host(out), g[f"dst{i}"]), i
        i += 1


@pytest.mark.parametrize("src,dst", [((1024, 1024), (512, 512)), ((2048, 2048), (1024, 1024)), ((128, 96), (64, 48)),
                                     ((37, 41), (19, 20)), ((64, 64), (32, 64)), ((40, 128), (40, 64)),
                                     ((64, 96), (128, 150)), ((512, 512), (16, 16)), ((1024, 1024), (128, 128)),
                                     ((1000, 760), (100, 95)), ((96, 1024), (12, 120)), ((8, 8192), (8, 128)),
                                     ((300, 40), (9, 40)), ((1024, 2048), (128, 256)), ((600, 1800), (60, 180))])
@pytest.mark.parametrize("bicubic", [True, False])
def test_resize_vs_oracle(torch_cuda, src, dst, bicubic):
    from ofb200 import ops
    a = rng(3).uniform(0, 255, src).astype(np.float32)
    out = ops.resize(dev(torch_cuda, a), (dst[1], dst[0]), bicubic)
    assert np.array_equal(host(out), O.resize(a, (dst[1], dst[0]), 1 if bicubic else 0))


def test_spline_golden(torch_cuda):
    from ofb200 import ops
    g = golden("spline")
    i = 0
    while f"src{i}" in g:
        ref = g[f"dst{i}"]
        out = host(ops.spline_upsample(dev(torch_cuda, g[f"src{i}"]), *ref.shape))
        assert np.all(np.abs(out - ref) <= np.spacing(np.abs(ref).astype(np.float32))), i
        assert np.array_equal(out, O.spline_upsample(g[f"src{i}"], *ref.shape)), i
        i += 1


@pytest.mark.parametrize("h,w", [(512, 512), (64, 128), (4, 4), (5, 9)])
def test_spline_vs_oracle_scaled(torch_cuda, h, w):
    from ofb200 import ops
    a = rng(4).normal(0, 2, (h, w)).astype(np.float32)
    out = host(ops.spline_upsample(dev(torch_cuda, a), 2 * h, 2 * w, 2.0))
    assert np.array_equal(out, O.spline_upsample(a, 2 * h, 2 * w) * np.float32(2.0))


@pytest.mark.parametrize("h,w,H,W", [(512, 512, 1024, 1024), (64, 128, 128, 256), (4, 4, 8, 8), (5, 9, 11, 17),
                                     (37, 50, 75, 101)])
def test_spline_pair_equals_single(torch_cuda, h, w, H, W):
    """Both components in the same launches give the single-plane results bit for bit
    (and the oracle's), with different scales per component."""
    from ofb200 import ops
    r = rng(h + w)
    a = r.normal(0, 2, (h, w)).astype(np.float32)
    b = r.normal(0, 2, (h, w)).astype(np.float32)
    su, sv = np.float32(W / w), np.float32(H / h)
    ou, ov = ops.spline_upsample_pair(dev(torch_cuda, a), dev(torch_cuda, b), H, W, su, sv)
    assert np.array_equal(host(ou), host(ops.spline_upsample(dev(torch_cuda, a), H, W, su)))
    assert np.array_equal(host(ov), host(ops.spline_upsample(dev(torch_cuda, b), H, W, sv)))
    assert np.array_equal(host(ov), O.spline_upsample(b, H, W) * sv)


def test_warp_golden(torch_cuda):
    from ofb200 import ops
    g = golden("warp")
    d = lambda k: dev(torch_cuda, g[k])
    O0, O1 = ops.warp_pair(d("I0"), d("I1"), d("U"), d("V"))
    assert np.array_equal(host(O0), g["O0"]) and np.array_equal(host(O1), g["O1"])


# ------------------------------------------------------------------------------ A6/A7
def test_hs_golden(torch_cuda):
    from ofb200 import ops
    g = golden("hs")
    d = lambda k: dev(torch_cuda, g[k])
    fx, fy, ft = ops.hs_derivatives(d("f0"), d("f1"))
    assert np.array_equal(host(fx), g["fx"]) and np.array_equal(host(fy), g["fy"])
    assert np.array_equal(host(ft), g["ft"])
    U, V, e = ops.hs_solve(d("f0"), d("f1"), d("U0").clone(), d("V0").clone(), float(g["alpha"]), int(g["niter"]))
    assert np.array_equal(host(U), g["U"]) and np.array_equal(host(V), g["V"])
    assert float(e.item()) == pytest.approx(float(g["err"]), rel=1e-6)


def test_hs_config1_vs_oracle(torch_cuda):
    """Horn-Schunck calibration PyHSchunck_Fs3_4 at 256x256 (600 sweeps, alpha 21)."""
    from ofb200 import ops, synthetic as S
    a, b, Ug, Vg = S.config_pair("hs256", seed=0)
    taps = O.prepare_gaussian_kernel(3.4, 3)
    fa, fb = O.prefilter_taps(a.astype(np.float32), taps), O.prefilter_taps(b.astype(np.float32), taps)
    z = np.zeros_like(fa)
    U, V, e = ops.hs_solve(dev(torch_cuda, fa), dev(torch_cuda, fb), dev(torch_cuda, z), dev(torch_cuda, z), 21, 600)
    Uo, Vo, eo = O.hs_solve(fa, fb, z, z, 21, 600)
    assert np.array_equal(host(U), Uo) and np.array_equal(host(V), Vo)
    assert float(e.item()) == pytest.approx(eo, rel=1e-9)


@pytest.mark.parametrize("shape,niter", [((16, 16), 1), ((57, 130), 9), ((300, 201), 13), ((40, 56), 4),
                                         ((130, 61), 6), ((12, 40), 5), ((1024, 1024), 7)])
def test_hs_shapes_vs_oracle(torch_cuda, shape, niter):
    """Horn-Schunck across tile edges, image borders ('mirror'), images smaller than one
    tile and sweep counts that end mid-pass (the blocked kernel runs 4 sweeps per launch;
    images under 16 pixels a side take the one-sweep kernel)."""
    from ofb200 import ops
    r = rng(shape[0] + 3 * shape[1] + niter)
    a = r.uniform(0, 255, shape).astype(np.float32)
    b = r.uniform(0, 255, shape).astype(np.float32)
    U0 = r.normal(0, 0.5, shape).astype(np.float32)
    V0 = r.normal(0, 0.5, shape).astype(np.float32)
    U, V, e = ops.hs_solve(dev(torch_cuda, a), dev(torch_cuda, b), dev(torch_cuda, U0), dev(torch_cuda, V0), 21, niter)
    Uo, Vo, eo = O.hs_solve(a, b, U0, V0, 21, niter)
    assert np.array_equal(host(U), Uo) and np.array_equal(host(V), Vo)
    assert float(e.item()) == pytest.approx(eo, rel=1e-9)


# ------------------------------------------------------------------------------ A8/A9
def test_ls_golden(torch_cuda):
    from ofb200 import ops
    g = golden("ls")
    d = lambda k: dev(torch_cuda, g[k])
    U, V, it, e = ops.ls_solve(d("f0"), d("f1"), d("U0").clone(), d("V0").clone(), float(g["h"]))
    assert np.array_equal(host(U), g["U"]) and np.array_equal(host(V), g["V"])
    assert int(it.item()) == 60
    assert float(e.item()) == pytest.approx(float(g["err"]), rel=1e-6)
    f0 = dev(torch_cuda, g["f0"] / np.max(g["f0"]))
    c = ops.ls_coefficients(f0, torch_cuda.zeros_like(f0), 10.0)
    assert np.array_equal(host(c[5]), g["B11"]) and np.array_equal(host(c[7]), g["B22"])


@pytest.mark.parametrize("n", [64, 512])
def test_ls_vs_oracle(torch_cuda, n):
    from ofb200 import ops, synthetic as S
    a, b, Ug, Vg = S.config_pair("fbls1024", seed=1, size=n)
    a, b = a.astype(np.float32), b.astype(np.float32)
    U0 = (Ug * 0.8).astype(np.float32)
    V0 = (Vg * 0.8).astype(np.float32)
    U, V, it, e = ops.ls_solve(dev(torch_cuda, a), dev(torch_cuda, b), dev(torch_cuda, U0), dev(torch_cuda, V0), 10)
    Uo, Vo, eo, ito = O.ls_solve(a, b, U0, V0, 10)
    assert int(it.item()) == ito
    assert np.array_equal(host(U), Uo) and np.array_equal(host(V), Vo)


@pytest.mark.parametrize("shape,maxnum", [((1, 9), 5), ((7, 5), 9), ((25, 57), 9), ((49, 113), 13),
                                           ((130, 171), 7), ((24, 56), 4), ((97, 1), 6)])
def test_ls_ragged_vs_oracle(torch_cuda, shape, maxnum):
    """Shapes that are not multiples of the 56 x 24 pass tile (odd widths, single rows and
    columns, images smaller than one tile) and sweep counts that end mid-pass."""
    from ofb200 import ops
    r = rng(sum(shape) + maxnum)
    a = r.uniform(1, 255, shape).astype(np.float32)
    b = r.uniform(1, 255, shape).astype(np.float32)
    U0 = r.normal(0, 0.5, shape).astype(np.float32)
    V0 = r.normal(0, 0.5, shape).astype(np.float32)
    U, V, it, e = ops.ls_solve(dev(torch_cuda, a), dev(torch_cuda, b), dev(torch_cuda, U0), dev(torch_cuda, V0), 10,
                               maxnum, 1e-30)
    Uo, Vo, eo, ito = O.ls_solve(a, b, U0, V0, 10, maxnum, 1e-30)
    assert int(it.item()) == ito == maxnum
    assert np.array_equal(host(U), Uo) and np.array_equal(host(V), Vo)
    assert float(e.item()) == pytest.approx(eo, rel=1e-9)


@pytest.mark.parametrize("tol", [1e-3, 1e-5, 1e-30])
def test_ls_stop_rule(torch_cuda, tol):
    """The device-side stop rule ends at the same sweep as the reference loop."""
    from ofb200 import ops
    r = rng(5)
    a = r.uniform(0, 255, (48, 40)).astype(np.float32)
    b = r.uniform(0, 255, (48, 40)).astype(np.float32)
    z = np.zeros_like(a)
    U, V, it, e = ops.ls_solve(dev(torch_cuda, a), dev(torch_cuda, b), dev(torch_cuda, z), dev(torch_cuda, z), 10, 60,
                               tol)
    Uo, Vo, eo, ito = O.ls_solve(a, b, z, z, 10, 60, tol)
    assert int(it.item()) == ito
    assert np.array_equal(host(U), Uo) and np.array_equal(host(V), Vo)
    assert float(e.item()) == pytest.approx(eo, rel=1e-9)


# ------------------------------------------------------------------------------ A10/A11
@pytest.mark.parametrize("hw,shape", [(13, (64, 72)), (5, (40, 33)), (15, (37, 50))])
def test_lk_vs_oracle(torch_cuda, hw, shape):
    import torch
    from ofb200 import ops, synthetic as S
    a, b, Ug, Vg = S.piv_pair(shape[0], shape[1], "lamb_oseen", seed=7, core_radius=15, density=0.08)
    a, b = a.astype(np.float32), b.astype(np.float32)
    U0 = (Ug * 0.5).astype(np.float32)
    V0 = (Vg * 0.5).astype(np.float32)
    U, V = dev(torch_cuda, U0), dev(torch_cuda, V0)
    st = torch.empty(shape, dtype=torch.uint8, device="cuda")
    er = torch.empty(shape, dtype=torch.float32, device="cuda")
    ops.lk_dense(dev(torch_cuda, a), dev(torch_cuda, b), U, V, hw, 5, (0, 0, 0, 0), st, er)
    Uo, Vo, sto, ero = O.lk_dense(a, b, U0, V0, hw, 5, want_status=True)
    assert np.array_equal(host(U), Uo) and np.array_equal(host(V), Vo)
    assert np.array_equal(host(st), sto) and np.array_equal(host(er), ero)


def test_lk_singular_keeps_input(torch_cuda):
    from ofb200 import ops
    a = np.full((32, 32), 7.0, np.float32)  # flat: det(A) = 0 everywhere
    U0 = rng(6).normal(0, 1, (32, 32)).astype(np.float32)
    U, V = dev(torch_cuda, U0), dev(torch_cuda, U0 * 2)
    ops.lk_dense(dev(torch_cuda, a), dev(torch_cuda, a), U, V)
    assert np.array_equal(host(U), U0) and np.array_equal(host(V), U0 * 2)


# ------------------------------------------------------------------------------ A12-A19
@pytest.fixture(scope="module")
def fb_inputs():
    from ofb200 import synthetic as S
    a, b, Ug, Vg = S.config_pair("fbls1024", seed=2, size=96)
    return a.astype(np.float32), b.astype(np.float32), Ug, Vg


def test_fb_kernels_vs_oracle(torch_cuda, fb_inputs):
    from ofb200 import ops
    a, b, Ug, Vg = fb_inputs
    H, W = a.shape
    g, xg, xxg, ig = O.farneback_poly_consts(7, 1.5)
    pc = ops.poly_consts(g, xg, xxg, ig, 7)
    RA = ops.fb_polyexp(dev(torch_cuda, a), pc)
    RB = ops.fb_polyexp(dev(torch_cuda, b), pc)
    assert np.array_equal(host(RA), O.fb_polyexp(a)) and np.array_equal(host(RB), O.fb_polyexp(b))
    for n, s in ((3, 0.0), (9, 1.0), (33, 4.95)):
        hk = O.fb_half_kernel(n, s)
        assert np.array_equal(host(ops.fb_blur(dev(torch_cuda, a), hk)), O.fb_blur(a, hk))
    fx, fy = Ug * 0.7, Vg * 0.7
    M = ops.fb_update_matrices(dev(torch_cuda, fx), dev(torch_cuda, fy), RA, RB)
    Mo = O.fb_update_matrices(fx, fy, host(RA), host(RB))
    assert np.array_equal(host(M), Mo)
    wk = O.fb_half_kernel(33, 4.95)
    Mb = ops.fb_blur(M, wk, planes=5)
    assert np.array_equal(host(Mb), O.fb_blur(Mo, wk, planes=5))
    assert np.array_equal(host(ops.fb_box5(M, 16)), O.fb_box5(Mo, 16))
    ux, uy = ops.fb_update_flow(Mb, H)
    uxo, uyo = O.fb_update_flow(host(Mb), H, W)
    assert np.array_equal(host(ux), uxo) and np.array_equal(host(uy), uyo)
    # fused iteration == blur5 -> updateFlow -> updateMatrices
    cx, cy = dev(torch_cuda, fx), dev(torch_cuda, fy)
    Mout = torch_cuda.empty_like(M)
    ops.fb_iteration(M, Mout, RA, RB, cx, cy, wk, True)
    assert np.array_equal(host(cx), uxo) and np.array_equal(host(cy), uyo)
    assert np.array_equal(host(Mout), O.fb_update_matrices(uxo, uyo, host(RA), host(RB)))


@pytest.mark.parametrize("n,sigma", [(3, 0.5), (9, 1.5), (15, 2.2), (33, 4.95)])
def test_fb_blur_interior_and_border_tiles(torch_cuda, n, sigma):
    """The Farneback blur on an image with interior tiles (no reflect mapping) and border
    tiles, for the specialised half widths (1, 4) and run-time ones, over 2 stacked planes."""
    from ofb200 import ops
    a = rng(n).uniform(0, 255, (2 * 300, 257)).astype(np.float32)
    hk = O.fb_half_kernel(n, sigma)
    assert np.array_equal(host(ops.fb_blur(dev(torch_cuda, a), hk, planes=2)), O.fb_blur(a, hk, planes=2))


@pytest.mark.parametrize("shape,polyN,sigma", [((37, 250), 7, 1.5), ((130, 491), 7, 1.5), ((257, 480), 5, 1.1),
                                               ((9, 1000), 5, 1.1), ((3, 17), 7, 1.5), ((61, 77), 3, 0.9)])
def test_fb_polyexp_shapes_vs_oracle(torch_cuda, shape, polyN, sigma):
    """The tiled expansion (polyN 5 and 7) across tile edges, image borders and both store
    paths (widths that are and are not multiples of 4), and the row kernel (other polyN)."""
    from ofb200 import ops
    a = rng(shape[0] * 7 + shape[1]).uniform(0, 255, shape).astype(np.float32)
    g, xg, xxg, ig = O.farneback_poly_consts(polyN, sigma)
    R = ops.fb_polyexp(dev(torch_cuda, a), ops.poly_consts(g, xg, xxg, ig, polyN))
    assert np.array_equal(host(R), O.fb_polyexp(a, polyN, sigma))


@pytest.mark.parametrize("shape,polyN,sigma", [((37, 250), 7, 1.5), ((130, 491), 7, 1.5), ((257, 480), 5, 1.1),
                                               ((9, 1000), 5, 1.1), ((3, 17), 7, 1.5), ((3, 3), 5, 1.1),
                                               ((24, 254), 7, 1.5), ((25, 481), 7, 1.5), ((1024, 1024), 7, 1.5)])
def test_fb_polyexp_blurred_vs_two_launches(torch_cuda, shape, polyN, sigma):
    """Blur (3 taps, reflect-101) fused into the expansion equals the blur kernel followed
    by the expansion kernel, and the oracle's blur then expansion, bit for bit: tiles whose
    rows lie inside the image and border tiles, the left, right, top and bottom reflections,
    widths at and beside the 240-column tile edge."""
    from ofb200 import ops
    a = rng(shape[0] * 5 + shape[1]).uniform(0, 255, shape).astype(np.float32)
    hk = O.fb_half_kernel(3, 0.0)
    g, xg, xxg, ig = O.farneback_poly_consts(polyN, sigma)
    pc = ops.poly_consts(g, xg, xxg, ig, polyN)
    d = dev(torch_cuda, a)
    fused = host(ops.fb_polyexp_blurred(d, hk, pc))
    assert np.array_equal(fused, host(ops.fb_polyexp(ops.fb_blur(d, hk), pc)))
    assert np.array_equal(fused, O.fb_polyexp(O.fb_blur(a, hk), polyN, sigma))


@pytest.mark.parametrize("kw", [{}, {"useGaussian": False}, {"polyN": 5, "polySigma": 1.1},
                                {"pyramidalLevels": 2}])
def test_farneback_compute_vs_oracle(torch_cuda, fb_inputs, kw):
    import Farneback_PyCL as F
    a, b, Ug, Vg = fb_inputs
    z = np.zeros_like(a)
    fb = F.Farneback_PyCL(**kw)
    U, V, e = fb.compute(a, b, z, z)
    Uo, Vo, _ = O.farneback(a, b, z, z, **kw)
    assert e == "Unknown"
    assert np.array_equal(U, Uo) and np.array_equal(V, Vo)


# ------------------------------------------------------------------------------ A5 driver
def test_pyramid_hs_golden(torch_cuda):
    import GenericPyramidalOpticalFlow as G
    import HornSchunck as HS
    g = golden("pyr_hs")
    U, V = G.genericPyramidalOpticalFlow(g["f0"], g["f1"], 3.4, HS.HSOpticalFlowAlgoAdapter([21], 600), 1, 1, None)
    assert np.array_equal(U, g["U"]) and np.array_equal(V, g["V"])


def test_pyramid_hs_ls_golden(torch_cuda):
    import GenericPyramidalOpticalFlow as G
    import HornSchunck as HS
    import PhysicsBasedOpticalFlowLiuShen as LS
    g = golden("pyr_hs_ls")
    U, V = G.genericPyramidalOpticalFlow(g["f0"], g["f1"], 3.4, HS.HSOpticalFlowAlgoAdapter([21, 45], 100), 2, 1,
                                         0.48, LS.LiuShenOpticalFlowAlgoAdapter(10))
    assert np.abs(U - g["U"]).max() <= 1e-5 and np.abs(V - g["V"]).max() <= 1e-5


def test_pyramid_lk_pyr2_vs_oracle(torch_cuda):
    """denseLK_Fs2_0_PyrLvls2 calibration on a 128x128 Lamb-Oseen pair."""
    import GenericPyramidalOpticalFlow as G
    import denseLucasKanade_PyCL as LK
    from ofb200 import synthetic as S
    a, b, Ug, Vg = S.config_pair("lk512", seed=3, size=128)
    a, b = a.astype(np.float32), b.astype(np.float32)
    U, V = G.genericPyramidalOpticalFlow(a, b, 2, LK.denseLucasKanade_PyCl(Niter=5, halfWindow=13), 2, 1, 0.48, None,
                                         warping=False)
    Uo, Vo = O.pyramid(a, b, 2, O.LK(5, 13), 2, 1, 0.48, None, warping=False)
    assert np.abs(U - Uo).max() <= TOL_PX and np.abs(V - Vo).max() <= TOL_PX


def test_pyramid_fb_ls_pyr2_vs_oracle(torch_cuda):
    """LiuSE_Farneback_Fs0_0_PyrLvls2 calibration on a 256x256 random-Fourier pair."""
    import GenericPyramidalOpticalFlow as G
    import Farneback_PyCL as F
    import PhysicsBasedOpticalFlowLiuShen as LS
    from ofb200 import synthetic as S
    a, b, Ug, Vg = S.config_pair("fbls1024", seed=4, size=256)
    a, b = a.astype(np.float32), b.astype(np.float32)
    U, V = G.genericPyramidalOpticalFlow(a, b, 0, F.Farneback_PyCL(), 2, 1, 0.48, LS.LiuShenOpticalFlowAlgoAdapter(10))
    Uo, Vo = O.pyramid(a, b, 0, O.FB(), 2, 1, 0.48, O.LS(10))
    assert np.abs(U - Uo).max() <= TOL_PX and np.abs(V - Vo).max() <= TOL_PX
    assert np.array_equal(U, Uo) and np.array_equal(V, Vo)
    assert S.epe(U, V, Ug, Vg, 16) <= S.epe(Uo, Vo, Ug, Vg, 16) + 1e-6


def test_pyramid_hs_pyr2_warp_vs_oracle(torch_cuda):
    """PyHSchunck_Fs3_4_PyrLvls2 calibration (bilinear warp at the second level)."""
    import GenericPyramidalOpticalFlow as G
    import HornSchunck as HS
    from ofb200 import synthetic as S
    a, b, Ug, Vg = S.config_pair("hs256", seed=5, size=128)
    a, b = a.astype(np.float32), b.astype(np.float32)
    U, V = G.genericPyramidalOpticalFlow(a, b, 3.4, HS.HSOpticalFlowAlgoAdapter([21, 45], 600), 2, 1, None)
    Uo, Vo = O.pyramid(a, b, 3.4, O.HS([21, 45], 600), 2)
    assert np.array_equal(U, Uo) and np.array_equal(V, Vo)


def test_torch_in_torch_out(torch_cuda):
    import GenericPyramidalOpticalFlow as G
    import HornSchunck as HS
    g = golden("pyr_hs")
    U, V = G.genericPyramidalOpticalFlow(dev(torch_cuda, g["f0"]), dev(torch_cuda, g["f1"]), 3.4,
                                         HS.HSOpticalFlowAlgoAdapter([21], 600), 1, 1, None)
    assert U.is_cuda and np.array_equal(host(U), g["U"])
