"""Drop-in for the reference's GenericPyramidalOpticalFlow module
(src/GenericPyramidalOpticalFlow.py): the coarse-to-fine driver that calls a main
optical-flow adapter and an optional refining adapter per pyramid level.

The whole pyramid runs on the GPU: the frames are uploaded once, each level's resize
(PIL BICUBIC semantics), flow upsample (RectBivariateSpline semantics), bilinear warp,
prefilter and the adapters' kernels run on the device, and U, V come back once.  Adapters
from this package are driven through their device path; any other object implementing
the reference's adapter protocol (compute / getAlgoName / hasGenericPyramidalDefaults /
getGenericPyramidalDefaults) is called with numpy arrays, exactly like the reference.

Both warps of the level transition are supported: bilinear (biLinear=True) and Liu-Shen's
optical-flow-equation warp (biLinear=False, :184-218), which, like the reference, edits
the level's first frame in place (the caller's frame at the last level) and raises
IndexError where the reference does.  Progress prints are off unless OFB200_VERBOSE=1.
"""
import numpy as np

from gaussian_filter import prepareGaussianKernel
from ofb200 import graph as _graph
from ofb200 import ops, to_device, is_host, to_host, to_host_pair, log, _torch

__all__ = ["genericPyramidalOpticalFlow", "updateNextPyramidalLevel", "doBiLinearWarping", "imresize"]


def imresize(im, res):
    """PIL BICUBIC resize of a float32 image to res = (width, height) (:66-67)."""
    host = is_host(im)
    out = ops.resize(to_device(im), res, bicubic=True)
    return to_host(out) if host else out


def doBiLinearWarping(img, coordsY, coordsX, order=1, mode='nearest'):
    """:69-115: img sampled at float32 (coordsY, coordsX), round-half-even base index."""
    host = is_host(img)
    out = ops.warp_coords(to_device(img), to_device(np.float32(coordsY) if host else coordsY),
                          to_device(np.float32(coordsX) if host else coordsX))
    return to_host(out) if host else out


def _prefilter(img, sigma, K):
    return ops.prefilter(img, prepareGaussianKernel(sigma, K))


def updateNextPyramidalLevel(im1IterNext, im1IterPrev, im2IterNext, Uaccum, Vaccum, U, V, warping=True,
                             biLinear=True, scale=False):
    """:117-234 on device tensors (numpy inputs are accepted and returned as numpy)."""
    host = is_host(im1IterNext)
    d = to_device
    n1, n2, Ua, Va = d(im1IterNext), d(im2IterNext), d(Uaccum), d(Vaccum)
    try:
        res = _transition(n1, tuple(im1IterPrev.shape), n2, Ua, Va, warping, biLinear, scale)
    finally:  # the Liu-Shen warp edits im1IterNext in place, as the reference does
        if warping and not biLinear and host and isinstance(im1IterNext, np.ndarray) \
                and im1IterNext.dtype == np.float32 and im1IterNext.flags.writeable:
            np.copyto(im1IterNext, to_host(n1))
    return tuple(to_host(t) for t in res) if host else res


def _transition(n1, prev_shape, n2, Ua, Va, warping, biLinear, scale):
    torch = _torch()
    H, W = n1.shape
    h, w = prev_shape
    sx = np.float32(np.float32(W) / np.float32(w)) if scale else np.float32(1.0)
    sy = np.float32(np.float32(H) / np.float32(h)) if scale else np.float32(1.0)
    if (h, w) != (H, W):
        if Ua.shape == Va.shape and Ua.stride(0) == Va.stride(0):
            us, vs = ops.spline_upsample_pair(Ua, Va, H, W, sx, sy)
        else:
            us = ops.spline_upsample(Ua, H, W, sx)
            vs = ops.spline_upsample(Va, H, W, sy)
    else:
        us = ops.scale(Ua, sx) if scale else Ua
        vs = ops.scale(Va, sy) if scale else Va
    if warping:
        if not biLinear:
            _liushen_warp(n1, us, vs)
            return n1, n2, us, vs, torch.zeros_like(n1), torch.zeros_like(n1)
        O0, O1 = ops.warp_pair(n1, n2, us, vs)
        return O0, O1, us, vs, torch.zeros_like(n1), torch.zeros_like(n1)
    return n1, n2, torch.zeros_like(n1), torch.zeros_like(n1), us, vs


# the warp's smoothing: gaussian_filter(d, 0.6 * mask_size, truncate=4.0 / 0.6 * mask_size)
# with mask_size 3 (:207-208), the reference's own separable filter (src/gaussian_filter.py:87-90)
_LSW_SIGMA = 0.6 * 3
_LSW_K = 2 * int(4.0 / 0.6 * 3 * _LSW_SIGMA + 0.5) + 1


def _liushen_warp(n1, us, vs):
    """:184-218 in place on n1: the integer scatter (IndexError beyond the image, as numpy
    reports it), the 73-tap smoothing of the sub-pixel parts (IndexError below 36 pixels),
    the optical-flow-equation correction.  Reads two ints back from the device."""
    H, W = n1.shape
    out, du, dv, bad = ops.warp_liushen_scatter(n1, us, vs)
    bv, bu = (int(b) for b in bad.cpu().tolist())
    for pos, axis, size, shift in ((bv, 0, H, vs), (bu, 1, W, us)):
        if pos != 2 ** 31 - 1:  # the first out-of-range index, row-major, axis 0 first
            y, x = divmod(pos, W)
            f = float(np.floor(np.float32(float(shift[y, x])) + np.float32(0.5)))
            idx = (y if axis == 0 else x) + int(f) if np.isfinite(f) else f
            raise IndexError(f"index {idx} is out of bounds for axis {axis} with size {size}")
    h = _LSW_K // 2
    if W < h or H < h:  # convolveSeparableFilter reads image[i, j] for j < K // 2
        n1.copy_(out)
        ax, sz = (1, W) if W < h else (0, H)
        raise IndexError(f"index {sz} is out of bounds for axis {ax} with size {sz}")
    taps = prepareGaussianKernel(_LSW_SIGMA, _LSW_K)
    n1.copy_(ops.warp_liushen_ofe(out, ops.prefilter(du, taps), ops.prefilter(dv, taps)))
    return n1


def _adapter_call(adapter, I0, I1, U, V):
    if hasattr(adapter, "_compute_dev"):
        return adapter._compute_dev(I0, I1, U, V)
    u, v, e = adapter.compute(to_host(I0), to_host(I1), to_host(U), to_host(V))
    return to_device(u), to_device(v), e


def genericPyramidalOpticalFlow(im1, im2, FILTER, mainOFlowAlgoAdapter, pyramidalLevels=1, kLevels=1,
                                FILTER_OPT=None, optionalOFlowAlgoAdapter=None, warping=True, biLinear=True,
                                pyramidalIntermediateScaling=True, pyramidalScaling=False):
    """:237-415.  Returns (Uaccum, Vaccum): numpy arrays for numpy input, CUDA tensors for
    tensor input.

    With this package's adapters the whole pyramid is captured once per configuration
    into a CUDA graph and replayed on later calls (ofb200.graph); the adapters' visible
    state changes exactly as in the reference (Horn-Schunck pops one alpha per level)."""
    host = is_host(im1)
    dev = getattr(mainOFlowAlgoAdapter, "device", None)
    if host:  # uploaded below: straight into the graph's inputs, or to_device on the eager path
        torch = _torch()
        a1 = np.ascontiguousarray(im1, np.float32)
        a2 = np.ascontiguousarray(im2, np.float32)
        if a1.ndim != 2 or a1.shape != a2.shape:
            raise ValueError("expected two 2-D images of one shape")
        gdev = dev or torch.device("cuda", torch.cuda.current_device())
        shape, devidx, dense = a1.shape, gdev.index, True
    else:
        I1 = to_device(im1, dev)
        I2 = to_device(im2, I1.device)
        shape, devidx, dense = tuple(I1.shape), I1.device.index, I1.stride(0) == I1.shape[1]
    if mainOFlowAlgoAdapter.hasGenericPyramidalDefaults():
        dm = mainOFlowAlgoAdapter.getGenericPyramidalDefaults()
        if dm is not None:
            if dm.get('warping') is not None:
                warping = dm.get('warping')
            if dm.get('biLinear') is not None:
                biLinear = dm.get('biLinear')
            if dm.get('intermediateScaling') is not None:
                pyramidalIntermediateScaling = dm.get('intermediateScaling')
            if dm.get('scaling') is not None:
                pyramidalScaling = dm.get('scaling')
    cfg = (float(FILTER), int(pyramidalLevels), int(kLevels), None if FILTER_OPT is None else float(FILTER_OPT),
           bool(warping), bool(biLinear), bool(pyramidalIntermediateScaling), bool(pyramidalScaling))
    main, opt = mainOFlowAlgoAdapter, optionalOFlowAlgoAdapter
    ncalls = int(pyramidalLevels) * int(kLevels)
    keyable = all(a is None or hasattr(a, "_graph_key") for a in (main, opt))
    mk = main._graph_key(ncalls) if keyable else None
    ok = opt._graph_key(ncalls) if keyable and opt is not None else None
    lswarp = bool(warping) and not bool(biLinear) and int(pyramidalLevels) * int(kLevels) > 1
    if keyable and mk is not None and (opt is None or ok is not None) and _graph.ENABLED and dense and not lswarp:
        key = ("pyramid", tuple(shape), devidx, cfg, mk, ok)
        m2 = main._graph_clone(ncalls)
        o2 = None if opt is None else opt._graph_clone(ncalls)

        def fn(a, b):
            return _pyramid_dev(a, b, cfg, m2._graph_clone(ncalls), None if o2 is None else o2._graph_clone(ncalls))

        Uacc, Vacc = _graph.CACHE.run(key, fn, [a1, a2] if host else [I1, I2], device=devidx)
        main._graph_consume(ncalls)
        if opt is not None:
            opt._graph_consume(ncalls)
        if host:
            return to_host_pair(Uacc, Vacc)
        return Uacc.clone(), Vacc.clone()
    if host:
        I1 = to_device(a1 if a1 is not im1 else im1, dev)
        I2 = to_device(a2, I1.device)
    try:
        Uacc, Vacc = _pyramid_dev(I1, I2, cfg, main, opt)
    finally:
        # the Liu-Shen warp edits the last level's first frame, the caller's im1, in place
        if lswarp and host and int(pyramidalLevels) > 1 and isinstance(im1, np.ndarray) \
                and im1.dtype == np.float32 and im1.flags.writeable:
            np.copyto(im1, to_host(I1))
    if host:
        return to_host(Uacc), to_host(Vacc)
    return Uacc, Vacc


def _pyramid_dev(I1, I2, cfg, mainOFlowAlgoAdapter, optionalOFlowAlgoAdapter):
    """The pyramid loop on device tensors (no host synchronisation for package adapters)."""
    torch = _torch()
    FILTER, pyramidalLevels, kLevels, FILTER_OPT, warping, biLinear, pyramidalIntermediateScaling, \
        pyramidalScaling = cfg
    scale = 1.0 / (2.0 ** (pyramidalLevels - 1))
    U = V = Uacc = Vacc = None
    work1 = None
    for level in range(1, pyramidalLevels + 1):
        lscale = pyramidalScaling if level == pyramidalLevels else pyramidalIntermediateScaling
        prev_shape = None if work1 is None else tuple(work1.shape)
        if scale < 1.0 and level != pyramidalLevels:
            size = (int(np.round(I1.shape[1] * scale)), int(np.round(I1.shape[0] * scale)))
            n1 = ops.resize(I1, size, bicubic=True)
            n2 = ops.resize(I2, size, bicubic=True)
        elif scale > 1.0:
            raise Exception('Invalid scale level: ' + str(scale))
        else:
            n1, n2 = I1, I2
        if level > 1:
            w1, w2, Uacc, Vacc, U, V = _transition(n1, prev_shape, n2, Uacc, Vacc, warping, biLinear, lscale)
        else:
            w1, w2 = n1, n2
            U = torch.zeros_like(n1)
            V = torch.zeros_like(n1)
            Uacc = torch.zeros_like(n1)
            Vacc = torch.zeros_like(n1)
        if FILTER > 1e-3:
            work1, work2 = _prefilter(w1, FILTER, 3), _prefilter(w2, FILTER, 3)
        else:
            work1, work2 = w1, w2
        if optionalOFlowAlgoAdapter is not None and FILTER_OPT is not None and FILTER_OPT > 1e-3:
            opt1, opt2 = _prefilter(n1, FILTER_OPT, 5), _prefilter(n2, FILTER_OPT, 5)
        elif optionalOFlowAlgoAdapter is not None:
            opt1, opt2 = n1, n2
        for k in range(kLevels):
            log('Level=', level, ' kIter=', k)
            if k > 0:
                if warping:  # on a copy of the level frame (:393)
                    w1, w2, Uacc, Vacc, U, V = _transition(n1.clone(), tuple(n1.shape), n2, Uacc, Vacc, warping,
                                                           biLinear, False)
                    if FILTER > 1:
                        work1, work2 = _prefilter(w1, FILTER, 3), _prefilter(w2, FILTER, 3)
                    else:
                        work1, work2 = w1, w2
                else:
                    work1, work2, Uacc, Vacc, U, V = _transition(work1, tuple(work1.shape), work2, Uacc, Vacc,
                                                                 warping, biLinear, False)
            U, V, error = _adapter_call(mainOFlowAlgoAdapter, work1, work2, U, V)
            if optionalOFlowAlgoAdapter is not None:
                U, V, errorOptional = _adapter_call(optionalOFlowAlgoAdapter, opt1, opt2, U, V)
            Uacc = ops.accumulate(Uacc.clone(), U)
            Vacc = ops.accumulate(Vacc.clone(), V)
        scale *= 2
    return Uacc, Vacc
