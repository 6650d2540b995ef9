"""The CPU oracle against golden vectors produced by the reference itself
(tests/golden/make_golden.py).  Bit-exact except the spline upsample (<= 1 float32 ulp)."""
import numpy as np
import pytest

import oracle as O
from conftest import golden


def test_prefilter_taps():
    g = golden("taps_prefilter")
    for i, (s, K) in enumerate(g["params"]):
        assert np.array_equal(O.prepare_gaussian_kernel(s, int(K)), g[f"k{i}"])


def test_bitexact_taps():
    g = golden("taps_bitexact")
    for i, (n, s) in enumerate(g["params"]):
        assert np.array_equal(O.gaussian_kernel_bitexact(int(n), s), g[f"k{i}"]), (n, s)


def test_farneback_consts():
    g = golden("fb_consts")
    for i in range(3):
        n, s = g[f"n{i}"]
        gg, xg, xxg, ig = O.farneback_poly_consts(int(n), s)
        assert np.array_equal(gg, g[f"g{i}"]) and np.array_equal(xg, g[f"xg{i}"])
        assert np.array_equal(xxg, g[f"xxg{i}"]) and np.array_equal(ig, g[f"ig{i}"])
    for i in range(4):
        n, s = g[f"halfp{i}"]
        assert np.array_equal(O.fb_half_kernel(int(n), s), g[f"half{i}"])


def test_prefilter():
    g = golden("prefilter")
    for i, (s, K) in enumerate([(3.4, 3), (2.0, 3), (0.48, 5)]):
        assert np.array_equal(O.prefilter(g["img"], s, K), g[f"out{i}"])


def test_hs():
    g = golden("hs")
    fx, fy, ft = O.hs_derivatives(g["f0"], g["f1"])
    assert np.array_equal(fx, g["fx"]) and np.array_equal(fy, g["fy"]) and np.array_equal(ft, g["ft"])
    U, V, e = O.hs_solve(g["f0"], g["f1"], g["U0"], g["V0"], float(g["alpha"]), int(g["niter"]))
    assert np.array_equal(U, g["U"]) and np.array_equal(V, g["V"])
    assert e == pytest.approx(float(g["err"]), rel=1e-6)


def test_ls():
    g = golden("ls")
    c = O.ls_coeffs(g["f0"], g["f1"], float(g["h"]))
    assert np.array_equal(c[5], g["B11"]) and np.array_equal(c[6], g["B12"]) and np.array_equal(c[7], g["B22"])
    U, V, e, it = O.ls_solve(g["f0"], g["f1"], g["U0"], g["V0"], float(g["h"]))
    assert np.array_equal(U, g["U"]) and np.array_equal(V, g["V"])
    assert e == pytest.approx(float(g["err"]), rel=1e-6)


def test_warp():
    g = golden("warp")
    O0, O1 = O.warp_pair(g["I0"], g["I1"], g["U"], g["V"])
    assert np.array_equal(O0, g["O0"]) and np.array_equal(O1, g["O1"])


def test_resize():
    g = golden("resize")
    i = 0
    while f"src{i}" in g:
        W, H, f = g[f"spec{i}"]
        out = O.resize(g[f"src{i}"], (int(W), int(H)), int(f))
        assert np.array_equal(out, g[f"dst{i}"]), i
        i += 1


def test_spline():
    g = golden("spline")
    i = 0
    while f"src{i}" in g:
        ref = g[f"dst{i}"]
        out = O.spline_upsample(g[f"src{i}"], *ref.shape)
        ulp = np.spacing(np.abs(ref).astype(np.float32))
        assert np.all(np.abs(out - ref) <= ulp), i
        i += 1


def test_pyramid_hs():
    g = golden("pyr_hs")
    U, V = O.pyramid(g["f0"], g["f1"], 3.4, O.HS([21], 600), 1)
    assert np.array_equal(U, g["U"]) and np.array_equal(V, g["V"])


def test_pyramid_hs_ls():
    g = golden("pyr_hs_ls")
    U, V = O.pyramid(g["f0"], g["f1"], 3.4, O.HS([21, 45], 100), 2, 1, 0.48, O.LS(10))
    assert np.abs(U - g["U"]).max() <= 1e-5 and np.abs(V - g["V"]).max() <= 1e-5


def test_liushen_warp_transition():
    """updateNextPyramidalLevel with biLinear=False: the warp alone is bit-exact on the
    reference's upsampled fields; the whole transition (spline within 1 ulp) to 1e-3."""
    g = golden("warp_liushen")
    for i in range(3):
        H, W, h, w, scale = (int(x) for x in g[f"spec_{i}"])
        out = O.liushen_warp(g[f"I1_{i}"].copy(), g[f"ua_{i}"], g[f"va_{i}"])
        assert np.array_equal(out, g[f"O1_{i}"]), i
        o1, o2, ua, va, u0, v0 = O._level_transition(g[f"I1_{i}"].copy(), (h, w), g[f"I2_{i}"], g[f"Ua_{i}"],
                                                     g[f"Va_{i}"], True, False, bool(scale))
        assert np.abs(ua - g[f"ua_{i}"]).max() <= 1e-5 and np.abs(o1 - g[f"O1_{i}"]).max() <= 1e-3, i
        assert np.array_equal(o2, g[f"I2_{i}"]) and not u0.any() and not v0.any()


def test_liushen_warp_index_errors():
    g = golden("warp_liushen")
    assert int(g["raises"]) == 1 and int(g["small_raises"]) == 1
    Ua = g["bad_Ua"]
    with pytest.raises(IndexError, match="out of bounds for axis 1 with size 8"):
        O.liushen_warp(g["bad_I1"].copy(), Ua, np.zeros_like(Ua))
    z = np.zeros((40, 30), np.float32)
    with pytest.raises(IndexError) as e:
        O.liushen_warp(np.ones((40, 30), np.float32), z, z)
    assert str(e.value) == str(g["small_msg"])


def test_pyramid_hs_liushen_warp_klevels():
    """HS without adapter defaults, the Liu-Shen warp, 2 levels x 2 iterations, LS refine;
    the caller's first frame is edited in place as in the reference."""
    g = golden("pyr_hs_lswarp")
    f0 = g["f0"].copy()
    U, V = O.pyramid(f0, g["f1"], 3.4, O.HS([21, 45, 33, 17], 50, provideGenericPyramidalDefaults=False), 2, 2, 0.48,
                     O.LS(10), True, False, True, True)
    assert np.abs(U - g["U"]).max() <= 1e-3 and np.abs(V - g["V"]).max() <= 1e-3
    assert np.abs(f0 - g["f0_after"]).max() <= 1e-3 * np.abs(g["f0_after"]).max()


def test_prefilter_reference_errors():
    """The drop-in raises what the reference's gaussian_filterPx raises (before any GPU
    work): IndexError below half the kernel (columns checked first), ValueError for K == 1
    or an even K."""
    import gaussian_filter as GF
    g = golden("prefilter_errors")
    for i in range(6):
        H, W, K = (int(x) for x in g[f"case{i}"])
        want = str(g[f"msg{i}"])
        if not want:
            continue
        with pytest.raises((IndexError, ValueError)) as e:
            GF._reference_errors(K, H, W)
        assert f"{type(e.value).__name__}: {e.value}" == want, i
