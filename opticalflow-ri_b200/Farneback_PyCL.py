"""Drop-in for the reference's Farneback_PyCL module (src/Farneback_PyCL.py): OpenCV's
Farneback dense flow on the GPU.  Every kernel call stays on the device (the reference
copies each buffer host<->device per kernel call); one solver iteration is one fused
kernel (blur5 -> updateFlow -> updateMatrices).

Same constructor and compute() as the reference; platformID is accepted and ignored,
deviceID selects the CUDA device.  The per-kernel methods (gaussianBlur, polynomialExpansion,
updateMatrices, ...) are kept with the reference's signatures and accept numpy arrays or
CUDA tensors.
"""
import functools

import numpy as np

from GaussianKernelBitExact import getGaussianKernelBitExact
from ofb200 import device_of, ops, to_device, is_host, to_host, _torch, log

__all__ = ["Farneback_PyCL", "imresize"]


def imresize(im, res):
    """PIL BILINEAR resize of a float32 image (src/Farneback_PyCL.py:61-62) on the device."""
    host = is_host(im)
    out = ops.resize(to_device(im), res, bicubic=False)
    return to_host(out) if host else out


@functools.lru_cache(maxsize=64)
def _prepare_gaussian(n, sigma):
    """src/Farneback_PyCL.py:123-171: g, xg, xxg (2n+1 float32 taps) and invG[1,1], invG[0,3],
    invG[3,3], invG[5,5] of the 6x6 moment matrix (float64)."""
    if sigma < 1.19209289550781250000000000000000000e-7:
        sigma = n * 0.3
    g = np.zeros([2 * n + 1], dtype=np.float32)
    xg = np.zeros([2 * n + 1], dtype=np.float32)
    xxg = np.zeros([2 * n + 1], dtype=np.float32)
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
    return g, xg, xxg, invG[1, 1], invG[0, 3], invG[3, 3], invG[5, 5]


class Farneback_PyCL(object):
    def __init__(self, windowSize=33, Niters=5, polyN=7, polySigma=1.5, useGaussian=True, pyrScale=0.5,
                 pyramidalLevels=1, platformID=0, deviceID=0, provideGenericPyramidalDefaults=True):
        assert pyramidalLevels >= 1, 'Pyramidal levels must be greater or equal than 1'
        self.useDouble = False
        self.windowSize = windowSize
        self.numIters = Niters
        self.polyN = int(polyN)
        self.polySigma = polySigma
        self.useGaussianFilter = useGaussian
        self.pyramidalLevels = pyramidalLevels - 1
        self.fastPyramids = False
        self.pyrScale = pyrScale
        self.provideGenericPyramidalDefaults = provideGenericPyramidalDefaults
        if windowSize & 1 == 0:
            raise Exception('windowSize must be an odd value')
        if windowSize // 2 > 32:
            raise ValueError('windowSize must be <= 65')
        self.device = device_of(platformID, deviceID)
        log('Running on device: ' + str(self.device))
        self.setPolynomialExpansionConsts()

    # ---------------------------------------------------------------- host constants
    def FarnebackPrepareGaussian(self):
        """src/Farneback_PyCL.py:123-171 (memoised per (polyN, polySigma))."""
        g, xg, xxg, a, b, c, d = _prepare_gaussian(self.polyN, float(self.polySigma))
        return g.copy(), xg.copy(), xxg.copy(), a, b, c, d


    def setPolynomialExpansionConsts(self):
        n = self.polyN
        g, xg, xxg, a, b, c, d = self.FarnebackPrepareGaussian()
        self.matrixG = g[n:].reshape([1, n + 1]).copy()
        self.matrixXG = xg[n:].reshape([1, n + 1]).copy()
        self.matrixXXG = xxg[n:].reshape([1, n + 1]).copy()
        self.matrixIGD = np.array([a, b, c, d], dtype=np.float64)
        self.matrixIG = np.float32(self.matrixIGD)
        self._poly = ops.poly_consts(self.matrixG[0], self.matrixXG[0], self.matrixXXG[0], self.matrixIG, n)

    def getGaussianKernel(self, n, sigma):
        _, kernel_bitexact = getGaussianKernelBitExact(n, sigma)
        return np.float32(kernel_bitexact).reshape([1, n])

    def setGaussianBlurKernel(self, smoothSize, sigma):
        g = self.getGaussianKernel(smoothSize, sigma)
        self.matrixGKernel = np.ascontiguousarray(g[0, int(smoothSize / 2):], dtype=np.float32).reshape([1, -1])

    # ---------------------------------------------------------------- kernels (reference signatures)
    def _wrap(self, fn, host, *ts):
        out = fn(*ts)
        if host:
            return tuple(to_host(o) for o in out) if isinstance(out, tuple) else to_host(out)
        return out

    def gaussianBlur(self, src, kSizeHalf, dst=None):
        host = is_host(src)
        return self._wrap(lambda s: ops.fb_blur(s, self.matrixGKernel[0, :int(kSizeHalf) + 1], 1), host,
                          to_device(src, self.device))

    def gaussianBlur5(self, src, kSizeHalf, dst=None):
        host = is_host(src)
        return self._wrap(lambda s: ops.fb_blur(s, self.matrixGKernel[0, :int(kSizeHalf) + 1], 5), host,
                          to_device(src, self.device))

    def boxFilter5(self, src, kSizeHalf, dst=None):
        host = is_host(src)
        return self._wrap(lambda s: ops.fb_box5(s, int(kSizeHalf)), host, to_device(src, self.device))

    def polynomialExpansion(self, src, dst=None):
        host = is_host(src)
        return self._wrap(lambda s: ops.fb_polyexp(s, self._poly), host, to_device(src, self.device))

    def updateFlow(self, M, flowX, flowY):
        host = is_host(M)
        H = flowX.shape[0]
        return self._wrap(lambda m: ops.fb_update_flow(m, H), host, to_device(M, self.device))

    def updateMatrices(self, flowX, flowY, RA, RB, M=None):
        host = is_host(flowX)
        d = lambda a: to_device(a, self.device)
        return self._wrap(ops.fb_update_matrices, host, d(flowX), d(flowY), d(RA), d(RB))

    def pyrDown(self, pyramid):
        raise Exception('Fast Pyramids not supported yet... Check ocl_pyrDown and ocl_pyrUp, pyrDown, pyrUp in OpenCV')

    # ---------------------------------------------------------------- driver
    def _compute_dev(self, im1, im2, U, V, consume_init=False):
        """src/Farneback_PyCL.py:461-603 on device tensors; returns (U, V, 'Unknown').
        consume_init: the caller hands U, V over (it does not read them afterwards), so a
        full-size first level iterates on them in place instead of on copies."""
        assert self.polyN == 5 or self.polyN == 7
        assert im1.shape == im2.shape and self.pyrScale < 1
        assert U.shape == im1.shape and V.shape == im1.shape
        size = im1.shape
        finalNumLevels = 0
        scale = 1
        while finalNumLevels < self.pyramidalLevels:
            scale *= self.pyrScale
            if size[1] * scale < 32 or size[0] * scale < 32:
                break
            finalNumLevels += 1
        prev = None
        cur = None
        for k in range(finalNumLevels, -1, -1):
            scale = 1.0
            for _ in range(k):
                scale *= self.pyrScale
            sigma = (1.0 / scale - 1.0) * 0.5
            smoothSize = max(int(round(sigma * 5)) | 1, 3)
            width, height = int(round(size[1] * scale)), int(round(size[0] * scale))
            if prev is None:
                cx = _scaled(ops.resize(U, (width, height), bicubic=False, copy=not consume_init), scale)
                cy = _scaled(ops.resize(V, (width, height), bicubic=False, copy=not consume_init), scale)
            else:
                cx = _scaled(ops.resize(prev[0], (width, height), bicubic=False), 1.0 / self.pyrScale)
                cy = _scaled(ops.resize(prev[1], (width, height), bicubic=False), 1.0 / self.pyrScale)
            self.setGaussianBlurKernel(smoothSize, sigma)
            gk = self.matrixGKernel[0]
            if ((height, width) == tuple(size) and len(gk) == 2 and min(size) >= 3 and im1.is_contiguous()
                    and im2.is_contiguous()):
                # full-size level, 3-tap blur: blur and expansion in one launch
                RA = ops.fb_polyexp_blurred(im1, gk, self._poly)
                RB = ops.fb_polyexp_blurred(im2, gk, self._poly)
            else:
                # the blurred frame is only read by the expansion: no copy at the full-size level
                RA = ops.fb_polyexp(ops.resize(ops.fb_blur(im1, gk, 1), (width, height), bicubic=False, copy=False),
                                    self._poly)
                RB = ops.fb_polyexp(ops.resize(ops.fb_blur(im2, gk, 1), (width, height), bicubic=False, copy=False),
                                    self._poly)
            M = ops.fb_update_matrices(cx, cy, RA, RB)
            if self.useGaussianFilter:
                self.setGaussianBlurKernel(self.windowSize, self.windowSize / 2 * 0.3)
                wk = self.matrixGKernel[0]
                Mb = torch_empty_like(M) if self.numIters > 1 else None
                for i in range(self.numIters):
                    upd = i < self.numIters - 1
                    ops.fb_iteration(M, Mb, RA, RB, cx, cy, wk, upd)
                    if upd:
                        M, Mb = Mb, M
            else:
                kh = int(self.windowSize / 2)
                for i in range(self.numIters):
                    Mb = ops.fb_box5(M, kh)
                    cx, cy = ops.fb_update_flow(Mb, height, cx, cy)
                    if i < self.numIters - 1:
                        M = ops.fb_update_matrices(cx, cy, RA, RB, M)
            prev = (cx, cy)
        return cx, cy, 'Unknown'

    def compute(self, im1, im2, U, V):
        host = is_host(im1)
        d = lambda a: to_device(a, self.device)
        Ud, Vd, e = self._compute_dev(d(im1), d(im2), d(U), d(V))
        if host:
            return to_host(Ud), to_host(Vd), e
        return Ud, Vd, e

    def _graph_key(self, n):
        return ("FB", self.windowSize, self.numIters, self.polyN, float(self.polySigma), bool(self.useGaussianFilter),
                float(self.pyrScale), self.pyramidalLevels, str(self.device))

    def _graph_clone(self, n):
        return self

    def _graph_consume(self, n):
        pass

    def getAlgoName(self):
        return 'Farneback CL'

    def hasGenericPyramidalDefaults(self):
        return self.provideGenericPyramidalDefaults

    def getGenericPyramidalDefaults(self):
        return {'warping': False, 'scaling': True}


def _scaled(t, s):
    """t * s in float32 (src/Farneback_PyCL.py:530-539); a factor of exactly 1 (the
    full-size level) changes no value, so the multiplication is skipped there."""
    return t if float(np.float32(s)) == 1.0 else ops.scale(t, s)


def torch_empty_like(t):
    return _torch().empty_like(t)
