"""CPU oracle for the dense pyramidal optical-flow hot path.

TEST INFRASTRUCTURE ONLY.  Restates the reference (OpticalFlow-RI) on the CPU so the
CUDA product can be checked against it.  Only ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` may import this module; the product package
never does.

The per-pixel kernels live in ``of_oracle.c`` (built by ``oracle/Makefile`` into
``oracle/_build/liboforacle.so``); this module wraps them with ctypes and restates the
host-side pieces in Python:

* tap generators: ``prepare_gaussian_kernel`` (src/gaussian_filter.py:47-52),
  ``gaussian_kernel_bitexact`` (src/GaussianKernelBitExact.py:55-144),
  ``farneback_poly_consts`` (src/Farneback_PyCL.py:123-196);
* the Farneback level driver (src/Farneback_PyCL.py:461-603);
* the pyramid driver (src/GenericPyramidalOpticalFlow.py:237-415), with the level
  transition of :117-234.

The float64 restatement of the HS / LS pipelines, used to separate algorithmic error from
float32 rounding, is ``oracle_f64.py``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from decimal import Decimal

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboforacle.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the C restatement (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(_HERE, "of_oracle.c")
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        I, F, D = ctypes.c_int, ctypes.c_float, ctypes.c_double
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.ofo_prefilter.argtypes = [_f32p, I, I, _f32p, I]
        L.ofo_hs_derivatives.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, I, I]
        L.ofo_hs_solve.argtypes = [_f32p, _f32p, _f32p, _f32p, I, I, F, I, dp]
        L.ofo_ls_coeffs.argtypes = [_f32p, _f32p, I, I, F, _f32p]
        L.ofo_ls_sweep.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, I, I, F, _f64p]
        L.ofo_ls_solve.argtypes = [_f32p, _f32p, _f32p, _f32p, I, I, F, I, D, ip, dp]
        L.ofo_warp_pair.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, _f32p, I, I]
        L.ofo_resize_coeffs.argtypes = [I, I, I, ctypes.c_void_p, ctypes.c_void_p, I]
        L.ofo_resize_coeffs.restype = I
        L.ofo_resize.argtypes = [_f32p, I, I, _f32p, I, I, I]
        L.ofo_spline_upsample.argtypes = [_f32p, I, I, _f32p, I, I]
        L.ofo_fb_polyexp.argtypes = [_f32p, _f32p, I, I, I, _f32p, _f32p, _f32p, _f32p]
        L.ofo_fb_blur.argtypes = [_f32p, _f32p, I, I, I, _f32p, I]
        L.ofo_fb_box5.argtypes = [_f32p, _f32p, I, I, I]
        L.ofo_fb_update_matrices.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, I, I]
        L.ofo_fb_update_flow.argtypes = [_f32p, _f32p, _f32p, I, I]
        L.ofo_lk_dense.argtypes = [_f32p, _f32p, _f32p, _f32p, I, I, I, I, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_void_p]
        _lib = L
    return _lib


def _c32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


# ----------------------------------------------------------------------------- taps
def prepare_gaussian_kernel(sigma, K):
    """src/gaussian_filter.py:47-52 (float32 storage, float32 normalisation)."""
    kernel = np.zeros(K, dtype=np.float32)
    xs = np.arange(-K / 2, K / 2, 1, dtype=int)
    kernel[:] = 1.0 / np.sqrt(2.0 * np.pi * sigma ** 2) * np.exp(-xs ** 2 / (2.0 * sigma ** 2))
    kernel /= np.sum(kernel)
    return kernel


def gaussian_kernel_bitexact(n, sigma):
    """src/GaussianKernelBitExact.py:55-144: returns the float64 kernel of n taps."""
    fixed = {1: [1.0], 3: [0.25, 0.5, 0.25], 5: [0.0625, 0.25, 0.375, 0.25, 0.0625],
             7: [0.03125, 0.109375, 0.21875, 0.28125, 0.21875, 0.109375, 0.03125],
             9: [4 / 256, 13 / 256, 30 / 256, 51 / 256, 60 / 256, 51 / 256, 30 / 256, 13 / 256, 4 / 256]}
    if sigma <= 0 and n in fixed:
        return np.array(fixed[n], dtype=np.float64)
    sigx = Decimal(sigma) if sigma < 0 else Decimal(n) * Decimal("0.15") + Decimal("0.35")
    scale2 = Decimal("-0.125") / (sigx * sigx)
    half = (n - 1) // 2
    vals = []
    x = 1 - n
    s = Decimal("0.0")
    for _ in range(half):
        t = (Decimal(x * x) * scale2).exp()
        vals.append(t)
        s += t
        x += 2
    s = s * Decimal(2.0) + Decimal("1.0")
    if (n & 1) == 0:
        s += Decimal("1.0")
    mul = Decimal("1.0") / s
    out = [Decimal(0)] * n
    for i in range(half):
        out[i] = out[n - 1 - i] = vals[i] * mul
    out[half] = Decimal("1.0") * mul
    if (n & 1) == 0:
        out[half + 1] = out[half]
    return np.array([float(v) for v in out], dtype=np.float64)


def fb_half_kernel(n, sigma):
    """src/Farneback_PyCL.py:198-208: float32 half kernel (centre first)."""
    g = np.float32(gaussian_kernel_bitexact(n, sigma))
    return np.ascontiguousarray(g[n // 2:], dtype=np.float32)


def farneback_poly_consts(polyN, polySigma):
    """src/Farneback_PyCL.py:123-196: g, xg, xxg (polyN+1 taps each) and ig (float32 x4)."""
    n, sigma = polyN, polySigma
    if sigma < 1.1920928955078125e-7:
        sigma = n * 0.3
    g = np.zeros(2 * n + 1, np.float32)
    xg = np.zeros(2 * n + 1, np.float32)
    xxg = np.zeros(2 * n + 1, np.float32)
    s = np.float64(0.0)
    for x in range(-n, n + 1):
        g[x + n] = np.exp(-x * x / (2 * sigma * sigma))
        s += g[x + n]
    s = 1.0 / s
    for x in range(-n, n + 1):
        g[x + n] = np.float32(g[x + n] * s)
        xg[x + n] = np.float32(x * g[x + n])
        xxg[x + n] = np.float32(x * x * g[x + n])
    G = np.zeros((6, 6), np.float64)
    for y in range(-n, n + 1):
        for x in range(-n, n + 1):
            G[0, 0] += g[y + n] * g[x + n]
            G[1, 1] += g[y + n] * g[x + n] * x * x
            G[3, 3] += g[y + n] * g[x + n] * x * x * x * x
            G[5, 5] += g[y + n] * g[x + n] * x * x * y * y
    G[2, 2] = G[0, 3] = G[0, 4] = G[3, 0] = G[4, 0] = G[1, 1]
    G[4, 4] = G[3, 3]
    G[3, 4] = G[4, 3] = G[5, 5]
    invG = np.linalg.inv(G)
    ig = np.array([invG[1, 1], invG[0, 3], invG[3, 3], invG[5, 5]], np.float32)
    return (np.ascontiguousarray(g[n:]), np.ascontiguousarray(xg[n:]), np.ascontiguousarray(xxg[n:]), ig)


# ----------------------------------------------------------------------------- kernels
def prefilter(img, sigma, K):
    """gaussian_filterPx (returns a new array; the reference filters in place)."""
    out = _c32(img).copy()
    lib().ofo_prefilter(out, out.shape[0], out.shape[1], _c32(prepare_gaussian_kernel(sigma, K)), K)
    return out


def prefilter_taps(img, taps):
    out = _c32(img).copy()
    lib().ofo_prefilter(out, out.shape[0], out.shape[1], _c32(taps), len(taps))
    return out


def hs_derivatives(f0, f1):
    f0, f1 = _c32(f0), _c32(f1)
    H, W = f0.shape
    fx, fy, ft = (np.empty((H, W), np.float32) for _ in range(3))
    lib().ofo_hs_derivatives(f0, f1, fx, fy, ft, H, W)
    return fx, fy, ft


def hs_solve(f0, f1, U, V, alpha, niter):
    """HS() semantics via the adapter (f0 = frame t0).  Returns (U, V, error)."""
    f0, f1 = _c32(f0), _c32(f1)
    U, V = _c32(U).copy(), _c32(V).copy()
    err = ctypes.c_double()
    lib().ofo_hs_solve(f0, f1, U, V, f0.shape[0], f0.shape[1], float(np.float32(alpha)), int(niter),
                       ctypes.byref(err))
    return U, V, err.value


def ls_coeffs(im1, im2, h):
    im1, im2 = _c32(im1), _c32(im2)
    H, W = im1.shape
    c = np.empty((8, H, W), np.float32)
    lib().ofo_ls_coeffs(im1, im2, H, W, float(np.float32(h)), c)
    return c


def ls_solve(im1, im2, U, V, h, maxnum=60, tol=1e-8):
    """LiuShenOpticalFlowAlgoAdapter.compute semantics.  Returns (U, V, error, iters)."""
    im1, im2 = _c32(im1), _c32(im2)
    U, V = _c32(U).copy(), _c32(V).copy()
    it, err = ctypes.c_int(), ctypes.c_double()
    lib().ofo_ls_solve(im1, im2, U, V, im1.shape[0], im1.shape[1], float(np.float32(h)), int(maxnum), float(tol),
                       ctypes.byref(it), ctypes.byref(err))
    return U, V, err.value, it.value


def warp_pair(I0, I1, U, V):
    I0, I1, U, V = _c32(I0), _c32(I1), _c32(U), _c32(V)
    O0, O1 = np.empty_like(I0), np.empty_like(I1)
    lib().ofo_warp_pair(I0, I1, U, V, O0, O1, I0.shape[0], I0.shape[1])
    return O0, O1


BILINEAR, BICUBIC = 0, 1


def resize(img, size_wh, filt):
    """PIL Image.fromarray(f32).resize((W, H), filter) restated."""
    img = _c32(img)
    Wd, Hd = int(size_wh[0]), int(size_wh[1])
    out = np.empty((Hd, Wd), np.float32)
    lib().ofo_resize(img, img.shape[0], img.shape[1], out, Hd, Wd, int(filt))
    return out


def spline_upsample(src, H, W):
    src = _c32(src)
    out = np.empty((H, W), np.float32)
    lib().ofo_spline_upsample(src, src.shape[0], src.shape[1], out, int(H), int(W))
    return out


def fb_polyexp(src, polyN=7, polySigma=1.5):
    src = _c32(src)
    H, W = src.shape
    g, xg, xxg, ig = farneback_poly_consts(polyN, polySigma)
    out = np.empty((5 * H, W), np.float32)
    lib().ofo_fb_polyexp(src, out, H, W, polyN, g, xg, xxg, ig)
    return out


def fb_blur(src, half_kernel, planes=1):
    src = _c32(src)
    H = src.shape[0] // planes
    W = src.shape[1]
    out = np.empty_like(src)
    lib().ofo_fb_blur(src, out, H, W, planes, _c32(half_kernel), len(half_kernel) - 1)
    return out


def fb_box5(src, kh):
    src = _c32(src)
    H = src.shape[0] // 5
    out = np.empty_like(src)
    lib().ofo_fb_box5(src, out, H, src.shape[1], int(kh))
    return out


def fb_update_matrices(fx, fy, R0, R1):
    fx, fy, R0, R1 = _c32(fx), _c32(fy), _c32(R0), _c32(R1)
    H, W = fx.shape
    M = np.empty((5 * H, W), np.float32)
    lib().ofo_fb_update_matrices(fx, fy, R0, R1, M, H, W)
    return M


def fb_update_flow(M, H, W):
    M = _c32(M)
    fx, fy = np.empty((H, W), np.float32), np.empty((H, W), np.float32)
    lib().ofo_fb_update_flow(M, fx, fy, H, W)
    return fx, fy


def farneback(im1, im2, U, V, windowSize=33, Niters=5, polyN=7, polySigma=1.5, useGaussian=True, pyrScale=0.5,
              pyramidalLevels=1):
    """Farneback_PyCL.compute (src/Farneback_PyCL.py:461-603).  Returns (U, V, 'Unknown')."""
    im1, im2 = _c32(im1), _c32(im2)
    Hs, Ws = im1.shape
    levels = pyramidalLevels - 1
    scale = 1.0
    nlev = 0
    while nlev < levels:
        scale *= pyrScale
        if Ws * scale < 32 or Hs * scale < 32:
            break
        nlev += 1
    g, xg, xxg, ig = farneback_poly_consts(polyN, polySigma)
    prev = None
    cur = None
    for k in range(nlev, -1, -1):
        scale = 1.0
        for _ in range(k):
            scale *= pyrScale
        sigma = (1.0 / scale - 1.0) * 0.5
        smooth = max(int(round(sigma * 5)) | 1, 3)
        width, height = int(round(Ws * scale)), int(round(Hs * scale))
        if prev is None:
            cx = resize(U, (width, height), BILINEAR) * np.float32(scale)
            cy = resize(V, (width, height), BILINEAR) * np.float32(scale)
        else:
            cx = resize(prev[0], (width, height), BILINEAR) * np.float32(1.0 / pyrScale)
            cy = resize(prev[1], (width, height), BILINEAR) * np.float32(1.0 / pyrScale)
        cx, cy = _c32(cx), _c32(cy)
        gk = fb_half_kernel(smooth, sigma)
        RA = np.empty((5 * height, width), np.float32)
        RB = np.empty((5 * height, width), np.float32)
        for src, R in ((im1, RA), (im2, RB)):
            bl = fb_blur(src, gk)
            lv = resize(bl, (width, height), BILINEAR)
            lib().ofo_fb_polyexp(_c32(lv), R, height, width, polyN, g, xg, xxg, ig)
        M = fb_update_matrices(cx, cy, RA, RB)
        wk = fb_half_kernel(windowSize, windowSize / 2 * 0.3)
        for i in range(Niters):
            if useGaussian:
                Mb = fb_blur(M, wk, planes=5)
            else:
                Mb = fb_box5(M, int(windowSize / 2))
            cx, cy = fb_update_flow(Mb, height, width)
            if i < Niters - 1:
                M = fb_update_matrices(cx, cy, RA, RB)
        prev = (cx, cy)
    return cx, cy, "Unknown"


def lk_dense(I, J, U, V, halfWindow=13, Niter=5, asym=(0, 0, 0, 0), want_status=False):
    """denseLucasKanade_PyCl.compute (src/denseLucasKanade_PyCL.py:113-169)."""
    I, J = _c32(I), _c32(J)
    U, V = _c32(U).copy(), _c32(V).copy()
    H, W = I.shape
    a = np.ascontiguousarray(asym, dtype=np.int32)
    st = np.ones((H, W), np.uint8)
    er = np.zeros((H, W), np.float32)
    lib().ofo_lk_dense(I, J, U, V, H, W, int(halfWindow), int(Niter), a.ctypes.data, st.ctypes.data,
                       er.ctypes.data)
    if want_status:
        return U, V, st, er
    return U, V, True


# ----------------------------------------------------------------------------- adapters
class HS:
    defaults = {"warping": True, "biLinear": True, "scaling": True}

    def __init__(self, alphas, Niter, provideGenericPyramidalDefaults=True):
        self.alphas, self.Niter = list(alphas), Niter
        if not provideGenericPyramidalDefaults:
            self.defaults = None

    def compute(self, im1, im2, U, V):
        return hs_solve(im1, im2, U, V, self.alphas.pop(), self.Niter)


class LS:
    defaults = None

    def __init__(self, alpha, maxnum=60, tol=1e-8):
        self.alpha, self.maxnum, self.tol = alpha, maxnum, tol
        self.iters = []

    def compute(self, im1, im2, U, V):
        u, v, e, it = ls_solve(im1, im2, U, V, self.alpha, self.maxnum, self.tol)
        self.iters.append(it)
        return u, v, e


class LK:
    defaults = {"warping": False, "intermediateScaling": True, "scaling": False}

    def __init__(self, Niter=5, halfWindow=13):
        self.Niter, self.halfWindow = Niter, halfWindow

    def compute(self, im1, im2, U, V):
        return lk_dense(im1, im2, U, V, self.halfWindow, self.Niter)


class FB:
    defaults = {"warping": False, "scaling": True}

    def __init__(self, **kw):
        self.kw = kw

    def compute(self, im1, im2, U, V):
        return farneback(im1, im2, U, V, **self.kw)


def liushen_warp(im1, us, vs):
    """The optical-flow-equation warp, in place on im1 (src/GenericPyramidalOpticalFlow.py:
    184-218): numpy's scatter (IndexError beyond the image, negative destinations wrap,
    the last source in row-major order wins), the sub-pixel parts smoothed by the
    reference's own 73-tap gaussian_filter (src/gaussian_filter.py:87-90, which raises
    IndexError below 36 pixels), then the float32 optical-flow-equation correction."""
    H, W = im1.shape
    ym, xm = np.meshgrid(np.arange(H, dtype=np.int32), np.arange(W, dtype=np.int32), indexing="ij")
    usSwap = np.int32(xm + np.floor(us + 0.5))
    vsSwap = np.int32(ym + np.floor(vs + 0.5))
    dU = us - np.floor(us + np.float32(0.5))
    dV = vs - np.floor(vs + np.float32(0.5))
    im1[vsSwap, usSwap] = im1[ym, xm]
    sigma, truncate = 0.6 * 3, 4.0 / 0.6 * 3
    K = 2 * int(truncate * sigma + 0.5) + 1
    h = K // 2
    for P in (dU, dV):
        if P.shape[1] < h:
            raise IndexError(f"index {P.shape[1]} is out of bounds for axis 1 with size {P.shape[1]}")
        if P.shape[0] < h:
            raise IndexError(f"index {P.shape[0]} is out of bounds for axis 0 with size {P.shape[0]}")
    taps = prepare_gaussian_kernel(sigma, K)
    dU, dV = prefilter_taps(dU, taps), prefilter_taps(dV, taps)
    tdx = im1[:-1, 1:] * dU[:-1, 1:] - im1[:-1, :-1] * dU[:-1, :-1]
    tdy = im1[1:, :-1] * dV[1:, :-1] - im1[:-1, :-1] * dV[:-1, :-1]
    im1[:-1, :-1] = im1[:-1, :-1] - (tdx + tdy)
    return im1


def _level_transition(im1_next, prev_shape, im2_next, Uacc, Vacc, warping, biLinear, scale):
    """src/GenericPyramidalOpticalFlow.py:117-234.  The Liu-Shen warp (biLinear=False)
    modifies im1_next in place, as the reference does."""
    H, W = im1_next.shape
    h, w = prev_shape
    if (h, w) != (H, W):
        us = spline_upsample(Uacc, H, W)
        vs = spline_upsample(Vacc, H, W)
    else:
        us, vs = Uacc.copy(), Vacc.copy()
    if scale:
        us *= np.float32(np.float32(W) / np.float32(w))
        vs *= np.float32(np.float32(H) / np.float32(h))
    if warping:
        if not biLinear:
            liushen_warp(im1_next, us, vs)
            z = np.zeros((H, W), np.float32)
            return im1_next, im2_next, us, vs, z, z.copy()
        O0, O1 = warp_pair(im1_next, im2_next, us, vs)
        z = np.zeros((H, W), np.float32)
        return O0, O1, us, vs, z, z.copy()
    z = np.zeros((H, W), np.float32)
    return im1_next, im2_next, z, z.copy(), us, vs


def pyramid(im1, im2, FILTER, main, pyramidalLevels=1, kLevels=1, FILTER_OPT=None, opt=None, warping=True,
            biLinear=True, pyramidalIntermediateScaling=True, pyramidalScaling=False):
    """genericPyramidalOpticalFlow (src/GenericPyramidalOpticalFlow.py:237-415)."""
    im1, im2 = _c32(im1), _c32(im2)
    d = main.defaults or {}
    warping = d.get("warping", warping)
    biLinear = d.get("biLinear", biLinear)
    pyramidalIntermediateScaling = d.get("intermediateScaling", pyramidalIntermediateScaling)
    pyramidalScaling = d.get("scaling", pyramidalScaling)
    scale = 1.0 / (2.0 ** (pyramidalLevels - 1))
    prev_shape = None
    U = V = Uacc = Vacc = None
    for level in range(1, pyramidalLevels + 1):
        lscale = pyramidalScaling if level == pyramidalLevels else pyramidalIntermediateScaling
        if scale < 1.0 and level != pyramidalLevels:
            size = (int(np.round(im1.shape[1] * scale)), int(np.round(im1.shape[0] * scale)))
            n1, n2 = resize(im1, size, BICUBIC), resize(im2, size, BICUBIC)
        else:
            n1, n2 = im1, im2
        if level > 1:
            w1, w2, Uacc, Vacc, U, V = _level_transition(n1, prev_shape, n2, Uacc, Vacc, warping, biLinear, lscale)
        else:
            w1, w2 = n1, n2
            U = np.zeros(n1.shape, np.float32)
            V = np.zeros(n1.shape, np.float32)
            Uacc = np.zeros(n1.shape, np.float32)
            Vacc = np.zeros(n1.shape, np.float32)
        if FILTER > 1e-3:
            k1, k2 = prefilter(w1, FILTER, 3), prefilter(w2, FILTER, 3)
        else:
            k1, k2 = w1.copy(), w2
        if opt is not None and FILTER_OPT is not None and FILTER_OPT > 1e-3:
            o1, o2 = prefilter(n1, FILTER_OPT, 5), prefilter(n2, FILTER_OPT, 5)
        elif opt is not None:
            o1, o2 = n1.copy(), n2
        prev_shape = k1.shape
        for k in range(kLevels):
            if k > 0:  # :391-403 (note FILTER > 1 here, FILTER > 1e-3 above)
                if warping:
                    w1, w2, Uacc, Vacc, U, V = _level_transition(n1.copy(), n1.shape, n2, Uacc, Vacc, warping,
                                                                 biLinear, False)
                    if FILTER > 1:
                        k1, k2 = prefilter(w1, FILTER, 3), prefilter(w2, FILTER, 3)
                    else:
                        k1, k2 = w1.copy(), w2
                else:
                    k1, k2, Uacc, Vacc, U, V = _level_transition(k1, k1.shape, k2, Uacc, Vacc, warping, biLinear,
                                                                 False)
            U, V, _ = main.compute(k1, k2, U, V)
            if opt is not None:
                U, V, _ = opt.compute(o1.copy(), o2.copy(), U, V)
            Uacc = Uacc + U
            Vacc = Vacc + V
        scale *= 2
    return Uacc, Vacc
