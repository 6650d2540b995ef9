"""Float64 restatement of the Horn-Schunck / Liu-Shen pyramid (TEST INFRASTRUCTURE ONLY).

The reference computes in float32 (its numba signatures are float32-only,
src/HornSchunck.py:51 and src/PhysicsBasedOpticalFlowLiuShen.py:75, and the examples cast
their frames to float32).  This module runs the same algorithms with the same code
structure in float64 throughout, so that the float32 GPU fields can be compared with the
algorithm's float64 answer (algorithmic error separated from float32 rounding):

* prefilter            src/gaussian_filter.py:24-94 (taps in float64, same border)
* imresize             src/GenericPyramidalOpticalFlow.py:66-67 (Pillow's antialiased
                       resample restated with a float64 intermediate)
* spline upsample      src/GenericPyramidalOpticalFlow.py:151-171 (scipy's
                       RectBivariateSpline itself, evaluated without the float32 cast)
* bilinear warp        src/GenericPyramidalOpticalFlow.py:69-115
* Horn-Schunck         src/HornSchunck.py:51-126 (scipy convolve on float64 planes)
* Liu-Shen             src/PhysicsBasedOpticalFlowLiuShen.py:33-158 (same)
* pyramid driver       src/GenericPyramidalOpticalFlow.py:237-415

Farneback has no float64 form here: the reference runs it in float32 OpenCL (its
USE_DOUBLE build is off, src/Farneback_PyCL.py:72); a Farneback main adapter runs the
float32 oracle and its output is widened to float64.
"""
from __future__ import annotations

import numpy as np
from scipy.interpolate import RectBivariateSpline
from scipy.ndimage import convolve

import oracle as O

f64 = lambda a: np.ascontiguousarray(a, np.float64)  # noqa: E731


def prepare_gaussian_kernel(sigma, K):
    """src/gaussian_filter.py:47-52 in float64."""
    x = np.arange(-K / 2, K / 2, 1, dtype=int).astype(np.float64)
    k = np.exp(-x * x / (2.0 * sigma * sigma))
    return k / k.sum()


def _prefilter_axis(img, k, axis):
    """One pass of convolveSeparableFilter (src/gaussian_filter.py:54-85): per line t is the
    line with h mirrored samples on the left and the last h samples copied in order on the
    right; out[x] = sum_j k[j] t[x+2h-j]."""
    a = np.moveaxis(img, axis, -1)
    n, K = a.shape[-1], len(k)
    h = K // 2
    if n < h:
        raise IndexError(f"index {n} is out of bounds for axis {axis} with size {n}")
    left = a[..., :h][..., ::-1]
    right = a[..., n - h:]
    t = np.concatenate([left, a, right], axis=-1)
    out = np.zeros_like(a)
    for j in range(K):
        out += k[j] * t[..., 2 * h - j:2 * h - j + n]
    return np.moveaxis(out, -1, axis)


def prefilter(img, sigma, K):
    k = prepare_gaussian_kernel(sigma, K)
    return _prefilter_axis(_prefilter_axis(f64(img), k, 1), k, 0)


def _resize_matrix(n_in, n_out, bicubic):
    """Pillow's antialiased resample weights (precompute_coeffs) as an n_out x n_in matrix."""
    def cubic(x):
        a = -0.5
        x = abs(x)
        if x < 1.0:
            return ((a + 2.0) * x - (a + 3.0)) * x * x + 1
        if x < 2.0:
            return (((x - 5) * x + 8) * x - 4) * a
        return 0.0

    def linear(x):
        x = abs(x)
        return 1.0 - x if x < 1.0 else 0.0

    f, fs = (cubic, 2.0) if bicubic else (linear, 1.0)
    scale = n_in / n_out
    fscale = max(scale, 1.0)
    support = fs * fscale
    Mx = np.zeros((n_out, n_in))
    for xx in range(n_out):
        center = (xx + 0.5) * scale
        xmin = max(int(center - support + 0.5), 0)
        xmax = min(int(center + support + 0.5), n_in)
        w = np.array([f((x - center + 0.5) / fscale) for x in range(xmin, xmax)])
        if w.sum() != 0:
            w = w / w.sum()
        Mx[xx, xmin:xmax] = w
    return Mx


def resize(img, size_wh, bicubic=True):
    img = f64(img)
    H, W = img.shape
    Wd, Hd = size_wh
    out = img
    if Wd != W:
        out = out @ _resize_matrix(W, Wd, bicubic).T
    if Hd != H:
        out = _resize_matrix(H, Hd, bicubic) @ out
    return out


def spline_upsample(src, H, W):
    h, w = src.shape
    ip = RectBivariateSpline(np.arange(h) / np.float32(h), np.arange(w) / np.float32(w), f64(src))
    return ip(np.arange(H) / np.float32(H), np.arange(W) / np.float32(W))


def bilinear_warp(img, cy, cx):
    """doBiLinearWarping (src/GenericPyramidalOpticalFlow.py:69-115) in float64."""
    H, W = img.shape
    iy, ix = np.round(cy).astype(np.int64), np.round(cx).astype(np.int64)
    dy, dx = cy - iy, cx - ix
    ny = np.where(dy < 0, iy - 1, iy + 1)
    nx = np.where(dx < 0, ix - 1, ix + 1)
    dy, dx = np.abs(dy), np.abs(dx)
    iy, ny = np.clip(iy, 0, H - 1), np.clip(ny, 0, H - 1)
    ix, nx = np.clip(ix, 0, W - 1), np.clip(nx, 0, W - 1)
    return ((1 - dy) * (1 - dx) * img[iy, ix] + (1 - dy) * dx * img[iy, nx] + dy * (1 - dx) * img[ny, ix]
            + dy * dx * img[ny, nx])


def warp_pair(I0, I1, U, V):
    H, W = I0.shape
    ym, xm = np.mgrid[0:H, 0:W].astype(np.float64)
    return bilinear_warp(f64(I0), ym - V / 2.0, xm - U / 2.0), bilinear_warp(f64(I1), ym + V / 2.0, xm + U / 2.0)


# ---- Horn-Schunck ------------------------------------------------------------------------
def hs_solve(im1, im2, U, V, alpha, niter):
    """HSOpticalFlowAlgoAdapter.compute -> HS(im1, im2, ...) (src/HornSchunck.py:34-104):
    HS names its first argument im2, so the derivatives are computeDerivatives(im2, im1)."""
    a, b = f64(im1), f64(im2)
    kx = np.array([[-1, 1], [-1, 1]], np.float64) * 0.25
    ky = np.array([[-1, -1], [1, 1]], np.float64) * 0.25
    kt = np.ones((2, 2), np.float64) * 0.25
    c = lambda x, k: convolve(x, k, mode="mirror")  # noqa: E731
    fx = c(b, kx) + c(a, kx)
    fy = c(b, ky) + c(a, ky)
    ft = c(a, kt) + c(b, -kt)
    kern = np.array([[1 / 12, 1 / 6, 1 / 12], [1 / 6, 0, 1 / 6], [1 / 12, 1 / 6, 1 / 12]], np.float64)
    u, v = f64(U), f64(V)
    den = alpha ** 2 + fx ** 2 + fy ** 2
    for _ in range(niter):
        ua, va = c(u, kern), c(v, kern)
        der = (fx * ua + fy * va + ft) / den
        u, v = ua - fx * der, va - fy * der
    err = (np.linalg.norm(u - U) + np.linalg.norm(v - V)) / (a.shape[0] * a.shape[1])
    return u, v, err


# ---- Liu-Shen ----------------------------------------------------------------------------
def ls_solve(im1, im2, U, V, h, maxnum=60, tol=1e-8):
    """LiuShenOpticalFlowAlgoAdapter.compute (src/PhysicsBasedOpticalFlowLiuShen.py:37-39):
    the solver's "u" is the row (y) component, so it is called with (V, U) and returns
    (resV, resU).  Returns (U, V, err, sweeps)."""
    I1, I2 = f64(im1), f64(im2)
    I1, I2 = I1 / I1.max(), I2 / I2.max()
    flip = lambda k: np.flipud(np.fliplr(k))  # noqa: E731
    D = flip(np.array([[0, -1, 0], [0, 0, 0], [0, 1, 0]], np.float64) / 2)
    M = flip(np.array([[1, 0, -1], [0, 0, 0], [-1, 0, 1]], np.float64) / 4)
    F = flip(np.array([[0, 1, 0], [0, 0, 0], [0, 1, 0]], np.float64))
    D2 = flip(np.array([[0, 1, 0], [0, -2, 0], [0, 1, 0]], np.float64))
    Hk = flip(np.array([[1, 1, 1], [1, 0, 1], [1, 1, 1]], np.float64))
    n = lambda x, k: convolve(x, k, mode="nearest")  # noqa: E731
    z = lambda x, k: convolve(x, k, mode="constant")  # noqa: E731
    IIx, IIy, II = I1 * n(I1, D), I1 * n(I1, D.T), I1 * I1
    Et = I2 - I1
    Ixt, Iyt = I1 * n(Et, D), I1 * n(Et, D.T)
    cm = z(np.ones_like(I1), Hk)
    A11 = I1 * (n(I1, D2) - 2 * I1) - h * cm
    A22 = I1 * (n(I1, D2.T) - 2 * I1) - h * cm
    A12 = I1 * n(I1, M)
    det = A11 * A22 - A12 * A12
    B11, B12, B22 = A22 / det, -A12 / det, A11 / det
    u, v = f64(V), f64(U)  # the solver's (row, column) components
    r, c = I1.shape
    k, err, total = 0, 0.0, 1e8
    while total > tol and k < maxnum:
        bu = (2 * IIx * n(u, D) + IIx * n(v, D.T) + IIy * n(v, D) + II * n(u, F) + II * n(v, M) + h * z(u, Hk)
              + Ixt)
        bv = (IIy * n(u, D) + IIx * n(u, D.T) + 2 * IIy * n(v, D.T) + II * n(u, M) + II * n(v, F.T) + h * z(v, Hk)
              + Iyt)
        un, vn = -(B11 * bu + B12 * bv), -(B12 * bu + B22 * bv)
        total = (np.linalg.norm(un - u) + np.linalg.norm(vn - v)) / (r * c)
        u, v, err, k = un, vn, total, k + 1
    return v, u, err, k


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


class FB:
    """Farneback in float32 (the reference has no float64 Farneback), widened to float64."""
    defaults = {"warping": False, "scaling": True}

    def __init__(self, **kw):
        self.kw = kw

    def compute(self, im1, im2, U, V):
        f = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731
        u, v, e = O.farneback(f(im1), f(im2), f(U), f(V), **self.kw)
        return f64(u), f64(v), e


def _transition(n1, prev_shape, n2, Uacc, Vacc, warping, scale):
    H, W = n1.shape
    h, w = prev_shape
    if (h, w) != (H, W):
        us, vs = spline_upsample(Uacc, H, W), spline_upsample(Vacc, H, W)
    else:
        us, vs = Uacc.copy(), Vacc.copy()
    if scale:
        us = us * (W / w)
        vs = vs * (H / h)
    z = np.zeros((H, W))
    if warping:
        w1, w2 = warp_pair(n1, n2, us, vs)
        return w1, w2, us, vs, z, z.copy()
    return n1, n2, z, z.copy(), us, vs


def pyramid(im1, im2, FILTER, main, pyramidalLevels=1, kLevels=1, FILTER_OPT=None, opt=None, warping=True,
            pyramidalIntermediateScaling=True, pyramidalScaling=False):
    """genericPyramidalOpticalFlow (src/GenericPyramidalOpticalFlow.py:237-415) in float64,
    bilinear-warp branch.  Returns (Uaccum, Vaccum) as float64."""
    im1, im2 = f64(im1), f64(im2)
    d = main.defaults or {}
    warping = d.get("warping", warping)
    if not d.get("biLinear", True):
        raise NotImplementedError("the optical-flow-equation warp has no float64 restatement")
    pyramidalIntermediateScaling = d.get("intermediateScaling", pyramidalIntermediateScaling)
    pyramidalScaling = d.get("scaling", pyramidalScaling)
    scale = 1.0 / (2.0 ** (pyramidalLevels - 1))
    prev_shape = None
    Uacc = Vacc = U = V = None
    for level in range(1, pyramidalLevels + 1):
        lscale = pyramidalScaling if level == pyramidalLevels else pyramidalIntermediateScaling
        if scale < 1.0 and level != pyramidalLevels:
            size = (int(np.round(im1.shape[1] * scale)), int(np.round(im1.shape[0] * scale)))
            n1, n2 = resize(im1, size), resize(im2, size)
        else:
            n1, n2 = im1, im2
        if level > 1:
            w1, w2, Uacc, Vacc, U, V = _transition(n1, prev_shape, n2, Uacc, Vacc, warping, lscale)
        else:
            w1, w2 = n1, n2
            U, V = np.zeros(n1.shape), np.zeros(n1.shape)
            Uacc, Vacc = np.zeros(n1.shape), np.zeros(n1.shape)
        k1, k2 = (prefilter(w1, FILTER, 3), prefilter(w2, FILTER, 3)) if FILTER > 1e-3 else (w1, w2)
        if opt is not None:
            o1, o2 = ((prefilter(n1, FILTER_OPT, 5), prefilter(n2, FILTER_OPT, 5))
                      if FILTER_OPT is not None and FILTER_OPT > 1e-3 else (n1, n2))
        prev_shape = k1.shape
        if kLevels != 1:
            raise NotImplementedError("kLevels > 1 has no float64 restatement")
        U, V, _ = main.compute(k1, k2, U, V)
        if opt is not None:
            U, V, _ = opt.compute(o1, o2, U, V)
        Uacc, Vacc = Uacc + U, Vacc + V
        scale *= 2
    return Uacc, Vacc
