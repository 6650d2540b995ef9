"""The CPU oracle's LK and Farneback restatement against the reference's own code.

Two sources, both from the reference itself (oracle/clref: its .cl kernel files compiled
for the host CPU with OpenCL's per-expression contraction, work-groups run as fibers with
real barriers, and an exact float32 bilinear sampler in place of the device's fixed-point
texture filter):

* golden fixtures made by running the reference's unmodified host modules
  (Farneback_PyCL.compute, denseLucasKanade_PyCl.compute, genericPyramidalOpticalFlow)
  on those kernels (tests/golden/make_golden_cl.py) -- no reference needed at test time;
* kernel-level calls into the compiled kernels themselves (oracle/_ref/, built from the
  reference tree by `make -C oracle/clref`), skipped where they were not built.

All comparisons are bit-exact.
"""
import numpy as np
import pytest

import clref
import oracle as O
from conftest import golden

f32 = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731


# ---- golden fixtures from the reference's host modules ------------------------------------
def test_lk_compute_matches_reference():
    g = golden("lk_ref")
    for i in range(int(g["n"])):
        hw, nit, vort = (int(x) for x in g[f"spec{i}"])
        asym = tuple(int(x) for x in g[f"asym{i}"]) if vort else (0, 0, 0, 0)
        U, V, ok = O.lk_dense(f32(g[f"I{i}"]), f32(g[f"J{i}"]), g[f"U0_{i}"], g[f"V0_{i}"], hw, nit, asym)
        assert ok is True
        assert np.array_equal(U, g[f"U{i}"]) and np.array_equal(V, g[f"V{i}"]), i


def test_lk_vorticity_cases_cover_both_windows():
    """The fixture's two rotation cases select the reference's two asymmetric windows."""
    g = golden("lk_ref")
    picked = {tuple(int(x) for x in g[f"asym{i}"]) for i in range(int(g["n"])) if int(g[f"spec{i}"][2])}
    assert picked == {(0, 1, 0, 1), (1, 0, 0, 1)}


def test_farneback_compute_matches_reference():
    g = golden("fb_ref")
    for i in range(int(g["n"])):
        ws, nit, pn, ps, ug, pl = g[f"spec{i}"]
        U, V, e = O.farneback(f32(g[f"I{i}"]), f32(g[f"J{i}"]), g[f"U0_{i}"], g[f"V0_{i}"], int(ws), int(nit), int(pn),
                              float(ps), bool(ug), 0.5, int(pl))
        assert e == "Unknown"
        assert np.array_equal(U, g[f"U{i}"]) and np.array_equal(V, g[f"V{i}"]), i


@pytest.mark.parametrize("name", ["pyr_lk_ref", "pyr_fb_ref", "pyr_fbls_ref"])
def test_pyramid_pipelines_match_reference(name):
    g = golden(name)
    a, b = f32(g["f0"]), f32(g["f1"])
    if name == "pyr_lk_ref":  # denseLK_Fs2_0_PyrLvls2 calibration
        U, V = O.pyramid(a, b, 2, O.LK(5, 13), 2, 1, 0.48, None, warping=False)[:2]
    elif name == "pyr_fb_ref":  # Farneback_Fs0_0_PyrLvls2 calibration
        U, V = O.pyramid(a, b, 0, O.FB(), 2, 1, None, None)[:2]
    else:  # LiuSE_Farneback_Fs0_0_PyrLvls2 calibration
        U, V = O.pyramid(a, b, 0, O.FB(), 2, 1, 0.48, O.LS(10))[:2]
    assert np.array_equal(U, g["U"]) and np.array_equal(V, g["V"])


# ---- kernel level, against the compiled reference kernels ---------------------------------
needs_ref = pytest.mark.skipif(not clref.available(), reason="oracle/_ref not built (needs the reference tree)")


@pytest.fixture(scope="module")
def frames():
    from ofb200 import synthetic as S
    a, b, _, _ = S.config_pair("fbls1024", seed=5, size=96)
    return f32(a), f32(b)


@needs_ref
@pytest.mark.parametrize("polyN,sigma", [(7, 1.5), (5, 1.1), (7, 0.0)])
@pytest.mark.parametrize("shape", [(96, 96), (37, 300), (8, 9)])
def test_kernel_polynomial_expansion(polyN, sigma, shape):
    rng = np.random.default_rng(polyN * 100 + shape[1])
    src = f32(rng.uniform(0, 255, shape))
    g, xg, xxg, ig = O.farneback_poly_consts(polyN, sigma)
    assert np.array_equal(clref.polyexp(src, polyN, g, xg, xxg, ig), O.fb_polyexp(src, polyN, sigma))


@needs_ref
@pytest.mark.parametrize("n,sigma", [(3, 0.5), (9, 1.5), (33, 4.95), (65, 10.0)])
def test_kernel_gaussian_blur(frames, n, sigma):
    gk = O.fb_half_kernel(n, sigma)
    assert np.array_equal(clref.blur(frames[0], gk, n // 2), O.fb_blur(frames[0], gk))
    M = f32(np.random.default_rng(n).normal(0, 3, (5 * 40, 70)))
    assert np.array_equal(clref.blur5(M, gk, n // 2), O.fb_blur(M, gk, planes=5))


@needs_ref
@pytest.mark.parametrize("kh", [1, 7, 16])
def test_kernel_box_filter(kh):
    M = f32(np.random.default_rng(kh).normal(0, 3, (5 * 33, 61)))
    assert np.array_equal(clref.box5(M, kh), O.fb_box5(M, kh))


@needs_ref
@pytest.mark.parametrize("spread", [0.3, 3.0, 40.0])
def test_kernel_update_matrices_and_flow(frames, spread):
    """Displacements from sub-pixel to far outside the image (the out-of-range branch)."""
    a, b = frames
    RA, RB = O.fb_polyexp(a), O.fb_polyexp(b)
    rng = np.random.default_rng(int(spread * 10))
    fx, fy = f32(rng.normal(0, spread, a.shape)), f32(rng.normal(0, spread, a.shape))
    M = clref.update_matrices(fx, fy, RA, RB)
    assert np.array_equal(M, O.fb_update_matrices(fx, fy, RA, RB))
    ux, uy = clref.update_flow(M)
    ox, oy = O.fb_update_flow(M, a.shape[0], a.shape[1])
    assert np.array_equal(ux, ox) and np.array_equal(uy, oy)


@needs_ref
@pytest.mark.parametrize("half_win,niter,asym,init", [
    (13, 5, (0, 0, 0, 0), 0.0), (13, 5, (0, 1, 0, 1), 0.8), (13, 5, (1, 0, 0, 1), 0.8), (5, 5, (0, 0, 0, 0), 0.8),
    (5, 3, (1, 0, 0, 1), 0.0), (13, 5, (0, 0, 0, 0), 25.0)])
def test_kernel_lk_dense(half_win, niter, asym, init):
    """lkDense with its status and per-pixel error, both window builds, both asymmetric
    windows, and initial flows that leave the image."""
    from ofb200 import synthetic as S
    a, b, _, _ = S.config_pair("lk512", seed=9, size=40)
    a, b = f32(a), f32(b)
    rng = np.random.default_rng(half_win + niter)
    U0 = f32(rng.normal(0, init, a.shape)) if init else np.zeros_like(a)
    V0 = f32(rng.normal(0, init, a.shape)) if init else np.zeros_like(a)
    ru, rv, rs, re = clref.lk_dense(a, b, U0, V0, half_win, niter, asym)
    ou, ov, os_, oe = O.lk_dense(a, b, U0, V0, half_win, niter, asym, want_status=True)
    assert np.array_equal(ru, ou) and np.array_equal(rv, ov)
    assert np.array_equal(rs, os_) and np.array_equal(re, oe)


@needs_ref
def test_contraction_matters():
    """Without contraction the reference's Farneback kernels round differently: the
    comparisons above are sensitive to the fused multiply-adds, not vacuous."""
    rng = np.random.default_rng(3)
    src = f32(rng.uniform(0, 255, (48, 64)))
    g, xg, xxg, ig = O.farneback_poly_consts(7, 1.5)
    assert not np.array_equal(clref.polyexp(src, 7, g, xg, xxg, ig, contract=False), O.fb_polyexp(src, 7, 1.5))
