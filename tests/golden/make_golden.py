"""Generates the golden fixtures in tests/golden/ from the reference implementation.

Run in a container that has the reference source tree (read-only); pass its src/
directory as the first argument or in REFERENCE_SRC:

    PYTHONDONTWRITEBYTECODE=1 NUMBA_CACHE_DIR=/tmp/numba python tests/golden/make_golden.py <reference>/src

The reference's CPU modules (gaussian_filter, GaussianKernelBitExact, HornSchunck,
PhysicsBasedOpticalFlowLiuShen, GenericPyramidalOpticalFlow) are imported as-is with
stubs for the plotting/debug modules they import at module level (matplotlib, IPython).
Farneback_PyCL is imported with a stub `pyopencl` to reach its host-side constant
generators only (FarnebackPrepareGaussian, getGaussianKernel); its OpenCL kernels are not
run.  Pillow and scipy provide the resize / spline outputs the reference calls.
Fixtures are small .npz files; the GPU box never reads the reference.
"""
from __future__ import annotations

import contextlib
import importlib
import io
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_SRC", "")
sys.dont_write_bytecode = True
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache_golden")
sys.path.insert(0, os.path.join(REPO, "opticalflow-ri_b200"))


def _stub_modules():
    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    for n in ("imshow", "figure", "show", "draw", "pause"):
        setattr(plt, n, lambda *a, **k: None)
    mpl.pyplot = plt
    ip = types.ModuleType("IPython")
    core = types.ModuleType("IPython.core")
    dbg = types.ModuleType("IPython.core.debugger")

    class Pdb:
        def set_trace(self, *a, **k):
            pass

    dbg.Pdb = Pdb
    core.debugger = dbg
    ip.core = core
    cl = types.ModuleType("pyopencl")
    cla = types.ModuleType("pyopencl.array")
    cl.array = cla
    for name, mod in (("matplotlib", mpl), ("matplotlib.pyplot", plt), ("IPython", ip), ("IPython.core", core),
                      ("IPython.core.debugger", dbg), ("pyopencl", cl), ("pyopencl.array", cla)):
        sys.modules.setdefault(name, mod)


def load_reference():
    if not REF or not os.path.isdir(REF):
        raise SystemExit("make_golden.py: give the reference's src/ directory (argument or REFERENCE_SRC)")
    _stub_modules()
    if REF not in sys.path:
        sys.path.insert(0, REF)
    names = ("gaussian_filter", "GaussianKernelBitExact", "HornSchunck", "PhysicsBasedOpticalFlowLiuShen",
             "GenericPyramidalOpticalFlow", "Farneback_PyCL")
    return {n: importlib.import_module(n) for n in names}


def quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


def main():
    from PIL import Image
    from scipy.interpolate import RectBivariateSpline

    from ofb200 import synthetic as S

    R = load_reference()
    rng = np.random.default_rng(20240607)
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    out = {}

    # --- taps: A1 prepareGaussianKernel, A14 getGaussianKernelBitExact, A13 polynomial constants
    pk = [(3.4, 3), (2.0, 3), (0.48, 5), (1.2, 7), (0.8, 9)]
    out["taps_prefilter"] = dict(params=np.array(pk), **{f"k{i}": R["gaussian_filter"].prepareGaussianKernel(s, K)
                                                      for i, (s, K) in enumerate(pk)})
    bx = [(3, 0), (5, 0), (7, 0), (9, 0), (1, 0), (3, 0.5), (5, 2.0), (11, 0), (13, 1.0), (33, 4.95), (21, 3.15),
          (15, -1.7)]
    out["taps_bitexact"] = dict(params=np.array(bx, dtype=np.float64),
                                **{f"k{i}": np.asarray(R["GaussianKernelBitExact"].getGaussianKernelBitExact(n, s)[1],
                                                       np.float64) for i, (n, s) in enumerate(bx)})
    FB = R["Farneback_PyCL"].Farneback_PyCL
    fbc = {}
    for i, (n, sg) in enumerate([(7, 1.5), (5, 1.1), (7, 0.0)]):
        obj = types.SimpleNamespace(polyN=n, polySigma=sg)
        g, xg, xxg, a, b, c, d = FB.FarnebackPrepareGaussian(obj)
        fbc[f"g{i}"], fbc[f"xg{i}"], fbc[f"xxg{i}"] = g[n:], xg[n:], xxg[n:]
        fbc[f"ig{i}"] = np.array([a, b, c, d], np.float32)
        fbc[f"n{i}"] = np.array([n, sg])
    for i, (n, sg) in enumerate([(33, 4.95), (3, 0.0), (9, 0.0), (17, 1.5)]):
        obj = types.SimpleNamespace()
        fbc[f"half{i}"] = FB.getGaussianKernel(obj, n, sg)[0, n // 2:]
        fbc[f"halfp{i}"] = np.array([n, sg])
    out["fb_consts"] = fbc

    # --- A1 prefilter
    img = f32(rng.uniform(0, 255, (37, 53)))
    d = {"img": img}
    for i, (s, K) in enumerate(pk[:3]):
        d[f"out{i}"] = R["gaussian_filter"].gaussian_filterPx(img.copy(), s, K)
    out["prefilter"] = d

    # --- A6/A7 HS
    a, b, Ug, Vg = S.piv_pair(48, 64, "poiseuille", seed=3)
    a, b = f32(a), f32(b)
    U0 = f32(rng.normal(0, 0.5, a.shape))
    V0 = f32(rng.normal(0, 0.5, a.shape))
    hs = R["HornSchunck"]
    fx, fy, ft = hs.computeDerivatives(b, a)
    ad = hs.HSOpticalFlowAlgoAdapter([21.3], 40)
    u, v, e = quiet(ad.compute, a, b, U0.copy(), V0.copy())
    out["hs"] = dict(f0=a, f1=b, U0=U0, V0=V0, alpha=np.float32(21.3), niter=40, fx=fx, fy=fy, ft=ft, U=u, V=v,
                     err=np.float64(e))

    # --- A8/A9 LS
    a, b, Ug, Vg = S.piv_pair(40, 56, "lamb_oseen", seed=4, core_radius=12)
    a, b = f32(a), f32(b)
    ls = R["PhysicsBasedOpticalFlowLiuShen"]
    ad = ls.LiuShenOpticalFlowAlgoAdapter(10)
    u, v, e = quiet(ad.compute, a, b, U0[:40, :56].copy(), V0[:40, :56].copy())
    B11, B12, B22 = ls.generate_invmatrix(a / np.max(a), np.float32(10), 1)
    out["ls"] = dict(f0=a, f1=b, U0=f32(U0[:40, :56]), V0=f32(V0[:40, :56]), h=np.float32(10), U=u, V=v,
                     err=np.float64(e), B11=B11, B12=B12, B22=B22)

    # --- A4 warp
    G = R["GenericPyramidalOpticalFlow"]
    H, W = 33, 47
    I0 = f32(rng.uniform(0, 255, (H, W)))
    I1 = f32(rng.uniform(0, 255, (H, W)))
    us = f32(rng.uniform(-6, 6, (H, W)))
    vs = f32(rng.uniform(-6, 6, (H, W)))
    us[0, :5] = [1.0, 3.0, -1.0, 2.5, -0.5]
    vs[1, :5] = [1.0, -3.0, 5.0, 0.5, -2.5]
    xm, ym = np.meshgrid(np.arange(W, dtype=np.int32), np.arange(H, dtype=np.int32))
    O0 = G.doBiLinearWarping(I0, np.float32(ym - vs / 2.0), np.float32(xm - us / 2.0), order=1, mode="nearest")
    O1 = G.doBiLinearWarping(I1, np.float32(ym + vs / 2.0), np.float32(xm + us / 2.0), order=1, mode="nearest")
    out["warp"] = dict(I0=I0, I1=I1, U=us, V=vs, O0=O0, O1=O1)

    # --- A2 resize (Pillow, mode F)
    d = {}
    cases = [((64, 96), (48, 32), "bicubic"), ((64, 96), (48, 32), "bilinear"), ((100, 70), (100, 35), "bicubic"),
             ((30, 40), (60, 80), "bicubic"), ((50, 50), (25, 25), "bilinear"), ((64, 64), (64, 64), "bicubic")]
    for i, (sh, dst, f) in enumerate(cases):
        src = f32(rng.uniform(0, 255, sh))
        flt = Image.BICUBIC if f == "bicubic" else Image.BILINEAR
        d[f"src{i}"] = src
        d[f"dst{i}"] = np.array(Image.fromarray(src).resize(dst, flt))
        d[f"spec{i}"] = np.array([dst[0], dst[1], 1 if f == "bicubic" else 0])
    out["resize"] = d

    # --- A3 spline upsample (RectBivariateSpline as called at :151-161)
    d = {}
    for i, (h, w, Hh, Ww) in enumerate([(16, 24, 32, 48), (5, 7, 10, 14), (4, 6, 8, 12), (33, 20, 66, 40),
                                        (32, 32, 64, 64)]):
        src = f32(rng.normal(0, 2, (h, w)))
        ip = RectBivariateSpline(np.arange(h) / np.float32(h), np.arange(w) / np.float32(w), src)
        d[f"src{i}"] = src
        d[f"dst{i}"] = np.float32(ip(np.arange(Hh) / np.float32(Hh), np.arange(Ww) / np.float32(Ww)))
    out["spline"] = d

    # --- A5 pyramid driver, full pipelines on small synthetic PIV pairs
    a, b, Ug, Vg = S.piv_pair(64, 64, "poiseuille", seed=5)
    a, b = f32(a), f32(b)
    Ur, Vr = quiet(G.genericPyramidalOpticalFlow, a, b, 3.4, hs.HSOpticalFlowAlgoAdapter([21], 600), 1, 1, None)
    out["pyr_hs"] = dict(f0=a, f1=b, U=Ur, V=Vr)
    a, b, Ug, Vg = S.piv_pair(64, 96, "lamb_oseen", seed=6, core_radius=20)
    a, b = f32(a), f32(b)
    Ur, Vr = quiet(G.genericPyramidalOpticalFlow, a, b, 3.4, hs.HSOpticalFlowAlgoAdapter([21, 45], 100), 2, 1, 0.48,
                   ls.LiuShenOpticalFlowAlgoAdapter(10))
    out["pyr_hs_ls"] = dict(f0=a, f1=b, U=Ur, V=Vr)

    out.update(liushen_warp_cases(R, rng))
    # the prefilter's own exceptions on images smaller than half the kernel, K = 1, even K
    d = {}
    for i, (shape, K) in enumerate([((1, 7), 3), ((5, 3), 9), ((3, 20), 9), ((7, 40), 15), ((6, 6), 1), ((6, 6), 4)]):
        try:
            R["gaussian_filter"].gaussian_filterPx(np.ones(shape, np.float32), 1.0, K)
            d[f"msg{i}"] = np.array("")
        except (IndexError, ValueError) as e:
            d[f"msg{i}"] = np.array(f"{type(e).__name__}: {e}")
        d[f"case{i}"] = np.array([shape[0], shape[1], K])
    out["prefilter_errors"] = d
    only = sys.argv[sys.argv.index("--only") + 1].split(",") if "--only" in sys.argv else None
    for name, d in out.items():
        if only and name not in only:
            continue
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **d)
        print("wrote", name, os.path.getsize(os.path.join(HERE, f"{name}.npz")))


def _in_bounds_field(rng, H, W, lo, hi):
    """Random displacements whose rounded destinations stay below the last row / column
    (the reference's scatter raises IndexError beyond them; negative ones wrap)."""
    us = np.float32(rng.uniform(lo, hi, (H, W)))
    vs = np.float32(rng.uniform(lo, hi, (H, W)))
    xm, ym = np.meshgrid(np.arange(W), np.arange(H))
    us = np.where(xm + np.floor(us + np.float32(0.5)) > W - 1, np.float32(W - 1 - xm) - np.float32(0.25), us)
    vs = np.where(ym + np.floor(vs + np.float32(0.5)) > H - 1, np.float32(H - 1 - ym) - np.float32(0.25), vs)
    return np.float32(us), np.float32(vs)


def liushen_warp_cases(R, rng):
    """The optical-flow-equation warp (biLinear=False, src/GenericPyramidalOpticalFlow.py:184-218)."""
    from ofb200 import synthetic as S
    G, hs, ls = R["GenericPyramidalOpticalFlow"], R["HornSchunck"], R["PhysicsBasedOpticalFlowLiuShen"]
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    out = {}
    # the level transition: same size, and upsampled from half size with scaling
    d = {}
    for i, (H, W, h, w, scale) in enumerate([(40, 48, 40, 48, False), (48, 56, 24, 28, True), (36, 36, 36, 36, False)]):
        I1 = f32(rng.uniform(0, 255, (H, W)))
        I2 = f32(rng.uniform(0, 255, (H, W)))
        if (h, w) == (H, W):
            Ua, Va = _in_bounds_field(rng, H, W, -3.0, 3.0)
        else:  # an accumulated field at half size whose upsampled, scaled copy stays in bounds
            Ua, Va = _in_bounds_field(rng, h, w, -0.7, 0.7)
            Ua = f32(np.where(np.arange(w)[None, :] >= w - 3, np.float32(-0.2), Ua))
            Va = f32(np.where(np.arange(h)[:, None] >= h - 3, np.float32(-0.2), Va))
        Z = np.zeros((h, w), np.float32)
        prev = np.zeros((h, w), np.float32)
        n1 = I1.copy()
        o1, o2, ua, va, u0, v0 = quiet(G.updateNextPyramidalLevel, n1, prev, I2, Ua.copy(), Va.copy(), Z, Z, True,
                                       False, scale)
        d.update({f"I1_{i}": I1, f"I2_{i}": I2, f"Ua_{i}": Ua, f"Va_{i}": Va, f"O1_{i}": o1, f"O2_{i}": o2,
                  f"ua_{i}": ua, f"va_{i}": va, f"spec_{i}": np.array([H, W, h, w, int(scale)])})
    # a destination beyond the last column raises IndexError in the reference
    I1 = f32(rng.uniform(0, 255, (8, 8)))
    Ua = np.zeros((8, 8), np.float32)
    Ua[3, 7] = 0.75
    try:
        quiet(G.updateNextPyramidalLevel, I1.copy(), I1, I1.copy(), Ua, np.zeros_like(Ua), Ua, Ua, True, False, False)
        d["raises"] = np.array(0)
    except IndexError:
        d["raises"] = np.array(1)
    d["bad_I1"], d["bad_Ua"] = I1, Ua
    # images smaller than the 73-tap filter's half width raise IndexError after the scatter
    I1 = f32(rng.uniform(0, 255, (40, 30)))
    n1 = I1.copy()
    Z = np.zeros_like(I1)
    try:
        quiet(G.updateNextPyramidalLevel, n1, I1, I1.copy(), Z, Z, Z, Z, True, False, False)
        d["small_raises"] = np.array(0)
    except IndexError as e:
        d["small_raises"] = np.array(1)
        d["small_msg"] = np.array(str(e))
    out["warp_liushen"] = d
    # full pipeline: HS (adapter defaults off) with the Liu-Shen warp, 2 levels, kLevels 2, LS refine
    for seed in range(20, 60):
        a, b, Ug, Vg = S.piv_pair(128, 128, "lamb_oseen", seed=seed, core_radius=12, max_disp=1.5)
        a, b = f32(a), f32(b)
        a_in = a.copy()
        try:
            Ur, Vr = quiet(G.genericPyramidalOpticalFlow, a_in, b, 3.4,
                           hs.HSOpticalFlowAlgoAdapter([21, 45, 33, 17], 50, provideGenericPyramidalDefaults=False), 2,
                           2, 0.48, ls.LiuShenOpticalFlowAlgoAdapter(10), True, False, True, True)
        except IndexError:
            continue
        out["pyr_hs_lswarp"] = dict(f0=a, f1=b, U=Ur, V=Vr, f0_after=a_in, seed=np.array(seed))
        break
    return out


if __name__ == "__main__":
    main()
