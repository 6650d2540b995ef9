"""Device-level operations: thin wrappers of the C ABI on torch CUDA tensors.

Every function takes and returns CUDA tensors (float32 planes, row-major, contiguous
rows; a plane may have a row pitch larger than its width), enqueues work on the current
torch stream and never synchronises.  Scratch memory comes from a per-(device, stream)
workspace cache.  torch provides device memory and streams only; all arithmetic runs in
libofb200.so.
"""
from __future__ import annotations

import contextlib
import ctypes
import os
import threading

import numpy as np
import torch

from . import _lib
from ._lib import FbPolyConsts, call, lib

__all__ = [
    "prefilter", "u8_to_f32", "resize", "spline_upsample", "spline_upsample_pair", "warp_pair", "accumulate", "scale", "hs_solve",
    "ls_solve", "lk_dense", "fb_blur", "fb_box5", "fb_polyexp", "fb_polyexp_blurred", "fb_update_matrices", "fb_update_flow",
    "fb_iteration", "workspace", "stream_ptr", "warp_liushen_scatter", "warp_liushen_ofe", "hs_batch", "hs_batch_shapes", "hs_batch_schedule",
]

_WS = {}
_RETIRED = []  # outgrown workspaces stay alive: captured CUDA graphs may still point at them


def stream_ptr():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def workspace(nbytes: int, slot: str = "main") -> tuple:
    """A device scratch buffer of >= nbytes for the current device and stream."""
    dev = torch.cuda.current_device()
    key = (dev, torch.cuda.current_stream().cuda_stream, slot)
    buf = _WS.get(key)
    if buf is None or buf.numel() < nbytes:
        if buf is not None:
            _RETIRED.append(buf)
        buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=f"cuda:{dev}")
        _WS[key] = buf
    return ctypes.c_void_p(buf.data_ptr()), ctypes.c_size_t(buf.numel())


def _plane(t: torch.Tensor, name: str, dtype=torch.float32):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name}: expected a CUDA tensor")
    if t.dtype != dtype:
        raise TypeError(f"{name}: expected {dtype}, got {t.dtype}")
    if t.dim() != 2 or t.stride(1) != 1:
        raise ValueError(f"{name}: expected a 2-D plane with contiguous rows")
    return ctypes.c_void_p(t.data_ptr()), t.shape[0], t.shape[1], t.stride(0)


def _new(H, W, like: torch.Tensor, dtype=torch.float32):
    return torch.empty((H, W), dtype=dtype, device=like.device)


def _same_pitch(*ts):
    p = ts[0].stride(0)
    for t in ts[1:]:
        if t.stride(0) != p or t.shape != ts[0].shape:
            raise ValueError("planes must share shape and row pitch")
    return p


# --------------------------------------------------------------------------- A1
def prefilter(src: torch.Tensor, taps, out: torch.Tensor | None = None) -> torch.Tensor:
    """Separable Gaussian prefilter (gaussian_filterPx semantics); src float32 or uint8."""
    taps = np.ascontiguousarray(taps, dtype=np.float32)
    H, W = src.shape
    out = _new(H, W, src) if out is None else out
    d, _, _, dp = _plane(out, "prefilter.out")
    if src.dtype == torch.uint8:
        s, _, _, sp = _plane(src, "prefilter.src", torch.uint8)
        call("of_prefilter_u8", s, sp, d, dp, H, W, taps.ctypes.data, len(taps), stream_ptr())
    else:
        s, _, _, sp = _plane(src, "prefilter.src")
        call("of_prefilter_f32", s, sp, d, dp, H, W, taps.ctypes.data, len(taps), stream_ptr())
    return out


def u8_to_f32(src: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """uint8 or uint16 (10/12-bit frames) plane -> float32 plane."""
    H, W = src.shape
    out = _new(H, W, src) if out is None else out
    d, _, _, dp = _plane(out, "u8_to_f32.out")
    if src.dtype == torch.uint16:
        s, _, _, sp = _plane(src, "u16_to_f32.src", torch.uint16)
        call("of_u16_to_f32", s, sp, d, dp, H, W, stream_ptr())
        return out
    s, _, _, sp = _plane(src, "u8_to_f32.src", torch.uint8)
    call("of_u8_to_f32", s, sp, d, dp, H, W, stream_ptr())
    return out


# --------------------------------------------------------------------------- A2/A3/A4
def resize(src: torch.Tensor, size_wh, bicubic: bool, out: torch.Tensor | None = None,
           copy: bool = True) -> torch.Tensor:
    """copy=False: a same-size resize returns `src` itself (for results that are only read,
    as the Farneback level's blurred frames are by the polynomial expansion)."""
    Wd, Hd = int(size_wh[0]), int(size_wh[1])
    if not copy and out is None and tuple(src.shape) == (Hd, Wd):
        return src
    s, Hs, Ws, sp = _plane(src, "resize.src")
    out = _new(Hd, Wd, src) if out is None else out
    d, _, _, dp = _plane(out, "resize.out")
    f = _lib.OF_FILTER_BICUBIC if bicubic else _lib.OF_FILTER_BILINEAR
    if max(_resize_taps(Ws, Wd, bicubic), _resize_taps(Hs, Hd, bicubic)) > RESIZE_TABLE_TAPS:
        th = _resize_table(Ws, Wd, f) if Wd != Ws else None
        tv = _resize_table(Hs, Hd, f) if Hd != Hs else None
        if (th is not None or Wd == Ws) and (tv is not None or Hd == Hs):
            ws, wn = workspace(4 * Hs * Wd, "resize")
            call("of_resize_tabled", s, Hs, Ws, sp, d, Hd, Wd, dp, f, None if th is None else _p(th),
                 None if tv is None else _p(tv), ws, wn, stream_ptr())
            return out
    ws, wn = workspace(lib().of_resize_workspace_size(Hs, Ws, Hd, Wd, f), "resize")
    call("of_resize", s, Hs, Ws, sp, d, Hd, Wd, dp, f, ws, wn, stream_ptr())
    return out


# Resizes with more taps per output than this (downscales by more than 4 with the bicubic
# filter, by more than 8 with the bilinear one) take their weights from tables computed
# once per (device, sizes, filter) and kept (of_resize_table), instead of recomputing them
# in every CTA.
RESIZE_TABLE_TAPS = 16
_RZ_TABLES = {}
_RZ_LOCK = threading.Lock()  # a table is built once even when host threads resize at once


def _resize_taps(n_in, n_out, bicubic):
    """Pillow's taps per output sample along one axis (the kernel's ksize)."""
    support = (2.0 if bicubic else 1.0) * max(n_in / n_out, 1.0)
    return int(np.ceil(support)) * 2 + 1


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _resize_table(n_in, n_out, f):
    """The weight table of one axis on the current device (None while a stream is being
    captured and the table does not exist yet: the caller then resizes without it)."""
    dev = torch.cuda.current_device()
    key = (dev, n_in, n_out, f)
    t = _RZ_TABLES.get(key)
    if t is None:
        if torch.cuda.is_current_stream_capturing():
            return None
        with _RZ_LOCK:
            t = _RZ_TABLES.get(key)
            if t is None:
                nb = lib().of_resize_table_size(n_in, n_out, f)
                t = torch.empty(nb, dtype=torch.uint8, device=f"cuda:{dev}")
                call("of_resize_table", n_in, n_out, f, _p(t), nb, stream_ptr())
                torch.cuda.current_stream().synchronize()  # later calls read it from any stream
                _RZ_TABLES[key] = t
    return t


def spline_upsample(src: torch.Tensor, H: int, W: int, scale: float = 1.0, out=None) -> torch.Tensor:
    s, h, w, sp = _plane(src, "spline.src")
    out = _new(H, W, src) if out is None else out
    d, _, _, dp = _plane(out, "spline.out")
    ws, wn = workspace(lib().of_spline_workspace_size(h, w, H, W), "spline")
    call("of_spline_upsample", s, h, w, sp, d, H, W, dp, float(np.float32(scale)), ws, wn, stream_ptr())
    return out


def spline_upsample_pair(su: torch.Tensor, sv: torch.Tensor, H: int, W: int, scale_u: float = 1.0,
                         scale_v: float = 1.0):
    """spline_upsample of both flow components in the same launches (bit-identical)."""
    s0, h, w, sp = _plane(su, "spline.src_u")
    s1, _, _, sp1 = _plane(sv, "spline.src_v")
    if sv.shape != su.shape or sp1 != sp:
        raise ValueError("spline_upsample_pair: the two components must share shape and pitch")
    ou, ov = _new(H, W, su), _new(H, W, su)
    d0, _, _, dp = _plane(ou, "spline.out_u")
    d1, _, _, dp1 = _plane(ov, "spline.out_v")
    if dp1 != dp:
        raise ValueError("spline_upsample_pair: output pitches differ")
    ws, wn = workspace(2 * lib().of_spline_workspace_size(h, w, H, W), "spline")
    call("of_spline_upsample_pair", s0, s1, h, w, sp, d0, d1, H, W, dp, float(np.float32(scale_u)),
         float(np.float32(scale_v)), ws, wn, stream_ptr())
    return ou, ov


def warp_pair(I0, I1, U, V):
    p = _same_pitch(I0, I1, U, V)
    H, W = I0.shape
    O0, O1 = torch.empty_like(I0), torch.empty_like(I1)
    call("of_warp_pair_bilinear", _plane(I0, "I0")[0], _plane(I1, "I1")[0], _plane(U, "U")[0], _plane(V, "V")[0],
         _plane(O0, "O0")[0], _plane(O1, "O1")[0], H, W, p, stream_ptr())
    return O0, O1


def warp_coords(img, coordsY, coordsX):
    p = _same_pitch(img, coordsY, coordsX)
    H, W = img.shape
    out = torch.empty_like(img)
    call("of_warp_bilinear_coords", _plane(img, "img")[0], _plane(coordsY, "coordsY")[0],
         _plane(coordsX, "coordsX")[0], _plane(out, "out")[0], H, W, p, stream_ptr())
    return out


def warp_liushen_scatter(I, us, vs):
    """Step 1 of the optical-flow-equation warp: (scattered image, du, dv, bad) with bad a
    device int32[2] (first out-of-range destination row / column position, INT_MAX)."""
    p = _same_pitch(I, us, vs)
    H, W = I.shape
    out, du, dv = torch.empty_like(I), torch.empty_like(I), torch.empty_like(I)
    bad = torch.empty(2, dtype=torch.int32, device=I.device)
    ws, wn = workspace(lib().of_warp_liushen_workspace_size(H, W), "lswarp")
    call("of_warp_liushen_scatter", _plane(I, "I")[0], _plane(us, "us")[0], _plane(vs, "vs")[0],
         _plane(out, "out")[0], _plane(du, "du")[0], _plane(dv, "dv")[0], H, W, p, ctypes.c_void_p(bad.data_ptr()),
         ws, wn, stream_ptr())
    return out, du, dv, bad


def warp_liushen_ofe(I, du, dv):
    """Step 3: the float32 optical-flow-equation correction of the scattered image."""
    p = _same_pitch(I, du, dv)
    H, W = I.shape
    out = torch.empty_like(I)
    call("of_warp_liushen_ofe", _plane(I, "I")[0], _plane(du, "du")[0], _plane(dv, "dv")[0], _plane(out, "out")[0],
         H, W, p, stream_ptr())
    return out


def accumulate(dst: torch.Tensor, src: torch.Tensor) -> torch.Tensor:
    p = _same_pitch(dst, src)
    H, W = dst.shape
    call("of_accumulate", _plane(dst, "dst")[0], _plane(src, "src")[0], H, W, p, stream_ptr())
    return dst


def scale(src: torch.Tensor, s: float, out=None) -> torch.Tensor:
    out = torch.empty_like(src) if out is None else out
    p = _same_pitch(src, out)
    H, W = src.shape
    call("of_scale", _plane(src, "src")[0], _plane(out, "out")[0], float(np.float32(s)), H, W, p, stream_ptr())
    return out


# --------------------------------------------------------------------------- A6/A7
_conc = threading.local()


@contextlib.contextmanager
def concurrent_streams():
    """Marks the work enqueued inside as running beside other streams' work (a multi-stream
    batch): solvers with a one-launch persistent form use their multi-launch form there,
    whose short launches interleave with the other streams."""
    _conc.depth = getattr(_conc, "depth", 0) + 1
    try:
        yield
    finally:
        _conc.depth -= 1


def in_concurrent_streams() -> bool:
    return getattr(_conc, "depth", 0) > 0


def hs_solve(I0, I1, U, V, alpha: float, niter: int, err: torch.Tensor | None = None, persistent=None):
    """Horn-Schunck in place on U, V.  Returns (U, V, err) with err a device float64 scalar.
    persistent: all sweeps in one launch (of_hs_solve_persistent) or one launch per pass of
    4 sweeps (of_hs_solve); None picks the persistent form except inside
    concurrent_streams().  Both give the same results bit for bit."""
    p = _same_pitch(I0, I1, U, V)
    H, W = I0.shape
    if persistent is None:
        persistent = not in_concurrent_streams()
    err = torch.empty((), dtype=torch.float64, device=I0.device) if err is None else err
    ws, wn = workspace(lib().of_hs_workspace_size(H, W, p), "hs")
    call("of_hs_solve_persistent" if persistent else "of_hs_solve", _plane(I0, "I0")[0], _plane(I1, "I1")[0],
         _plane(U, "U")[0], _plane(V, "V")[0], H, W, p, float(np.float32(alpha)), int(niter),
         ctypes.c_void_p(err.data_ptr()), ws, wn, stream_ptr())
    return U, V, err


def hs_derivatives(I0, I1):
    """fx, fy, ft of computeDerivatives(I1, I0) (I0 = frame t0, I1 = frame t1)."""
    p = _same_pitch(I0, I1)
    H, W = I0.shape
    fx, fy, ft = (torch.empty_like(I0) for _ in range(3))
    call("of_hs_derivatives", _plane(I0, "I0")[0], _plane(I1, "I1")[0], _plane(fx, "fx")[0], _plane(fy, "fy")[0],
         _plane(ft, "ft")[0], H, W, p, stream_ptr())
    return fx, fy, ft


# --------------------------------------------------------------------------- A8/A9
def ls_coefficients(I1n, Et, h: float):
    """The 8 Liu-Shen coefficient planes (IIx, IIy, II, Ixt, Iyt, B11, B12, B22) from a
    normalised frame and the normalised frame difference."""
    p = _same_pitch(I1n, Et)
    H, W = I1n.shape
    coef = torch.empty((8 * H, W), dtype=torch.float32, device=I1n.device)
    if coef.stride(0) != p:
        raise ValueError("ls_coefficients: planes must be unpadded")
    call("of_ls_coefficients", _plane(I1n, "I1n")[0], _plane(Et, "Et")[0], ctypes.c_void_p(coef.data_ptr()), H, W, p,
         float(np.float32(h)), stream_ptr())
    return coef.view(8, H, W)

LS_ARITHMETICS = ("fast", "exact")


def ls_arithmetic(arithmetic=None) -> str:
    """The Liu-Shen sweep's arithmetic: 'fast' (float32 with fused multiply-adds, within
    float32 rounding of the reference) or 'exact' (bit-exact with the reference's float32
    fields).  None reads OFB_LS_ARITHMETIC, default 'fast'."""
    a = arithmetic if arithmetic is not None else os.environ.get("OFB_LS_ARITHMETIC", "fast")
    if a not in LS_ARITHMETICS:
        raise ValueError(f"Liu-Shen arithmetic must be one of {LS_ARITHMETICS}, not {a!r}")
    return a


def ls_solve(I0, I1, U, V, h: float, maxnum: int = 60, tol: float = 1e-8, iters=None, err=None, arithmetic=None):
    """Liu-Shen in place on U (x) and V (y).  Returns (U, V, iters, err) (device scalars)."""
    p = _same_pitch(I0, I1, U, V)
    H, W = I0.shape
    mode = 1 if ls_arithmetic(arithmetic) == "fast" else 0  # OF_LS_FAST / OF_LS_EXACT
    iters = torch.empty((), dtype=torch.int32, device=I0.device) if iters is None else iters
    err = torch.empty((), dtype=torch.float64, device=I0.device) if err is None else err
    ws, wn = workspace(lib().of_ls_workspace_size(H, W, p, int(maxnum)), "ls")
    call("of_ls_solve_mode", _plane(I0, "I0")[0], _plane(I1, "I1")[0], _plane(U, "U")[0], _plane(V, "V")[0], H, W, p,
         float(np.float32(h)), int(maxnum), float(tol), mode, ctypes.c_void_p(iters.data_ptr()),
         ctypes.c_void_p(err.data_ptr()), ws, wn, stream_ptr())
    return U, V, iters, err


def hs_batch_shapes():
    """The persistent Horn-Schunck kernel's tile shapes: [(region_w, region_h, sweeps_per_pass)]."""
    out = []
    i = 0
    while True:
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        if lib().of_hs_batch_shape(i, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)) != 0:
            return out
        out.append((a.value, b.value, c.value))
        i += 1


HS_WAIT_LIMIT = 1 << 20  # polls of a queue wait before a pair is given up (under a second)


HS_SCHEDULES = ("auto", "queue", "resident", "cluster")  # OF_HS_SCHED_AUTO / _QUEUE / _RESIDENT / _CLUSTER


def hs_batch(pairs, tile_shape: int = 0, wait_limit: int = HS_WAIT_LIMIT, status=None, arithmetic: str = "exact",
             schedule: str = "auto"):
    """Horn-Schunck of many pairs in one persistent launch (of_hs_batch).  pairs: list of
    (I0, I1, U, V, alpha, niter) with CUDA float32 planes; U, V are updated in place.
    arithmetic: 'exact' (bit-exact with the reference) or 'fast' (float32 averaging).
    schedule: 'cluster' (one pair of at most 256 x 256 on one thread-block cluster, halos
    through distributed shared memory), 'resident' (one CTA per tile, region kept on chip;
    needs every tile to get a resident CTA), 'queue' (device work queue) or 'auto' (one CTA
    per tile when the device holds them, resident if they all run at once and the queue if
    not, decided on the device; else the queue; hs_batch_schedule tells which ran).
    Returns the per-pair status words (device int32, bits of ofb200._lib.ST_*)."""
    if arithmetic not in ("exact", "fast"):
        raise ValueError("arithmetic must be 'exact' or 'fast'")
    if schedule not in HS_SCHEDULES:
        raise ValueError(f"schedule must be one of {HS_SCHEDULES}")
    from ._lib import OfHsBatchPair, OfTuning
    n = len(pairs)
    arr = (OfHsBatchPair * n)()
    dev = pairs[0][0].device
    for k, (I0, I1, U, V, alpha, niter) in enumerate(pairs):
        p = _same_pitch(I0, I1, U, V)
        H, W = I0.shape
        arr[k] = OfHsBatchPair(I0.data_ptr(), I1.data_ptr(), U.data_ptr(), V.data_ptr(), H, W, p,
                               float(np.float32(alpha)), int(niter))
    if status is None:
        status = torch.zeros(n, dtype=torch.int32, device=dev)
    tun = OfTuning(int(tile_shape), 0, 1 if arithmetic == "fast" else 0, HS_SCHEDULES.index(schedule))
    ws, wn = workspace(lib().of_hs_batch_workspace_size(arr, n), "hs_batch")
    call("of_hs_batch", arr, n, ctypes.byref(tun), ctypes.c_void_p(status.data_ptr()), int(wait_limit), ws, wn,
         stream_ptr())
    return status


def _hs_batch_pairs(pairs):
    from ._lib import OfHsBatchPair
    arr = (OfHsBatchPair * len(pairs))()
    for k, (I0, I1, U, V, alpha, niter) in enumerate(pairs):
        H, W = I0.shape
        arr[k] = OfHsBatchPair(I0.data_ptr(), I1.data_ptr(), U.data_ptr(), V.data_ptr(), H, W, I0.stride(0),
                               float(np.float32(alpha)), int(niter))
    return arr


def hs_batch_schedule(pairs) -> str:
    """Which schedule the last hs_batch(pairs, schedule='auto') on this stream ran: 'resident'
    or 'queue' as its CTAs decided, or 'auto' when the launch chose statically (an explicit
    schedule, or more tiles than the device holds CTAs).  Synchronises the stream."""
    arr = _hs_batch_pairs(pairs)
    ws, wn = workspace(lib().of_hs_batch_workspace_size(arr, len(pairs)), "hs_batch")
    out = ctypes.c_int(-1)
    call("of_hs_batch_schedule", arr, len(pairs), ws, wn, ctypes.byref(out), stream_ptr())
    return HS_SCHEDULES[out.value]


# --------------------------------------------------------------------------- A10/A11
def lk_dense(I, J, U, V, half_win=13, niter=5, asym=(0, 0, 0, 0), status=None, err=None):
    """Dense LK in place on U, V.  status (uint8) / err (float32) planes are optional."""
    p = _same_pitch(I, J, U, V)
    H, W = I.shape
    a = np.ascontiguousarray(asym, dtype=np.int32)
    sp = ctypes.c_void_p(status.data_ptr()) if status is not None else None
    ep = ctypes.c_void_p(err.data_ptr()) if err is not None else None
    call("of_lk_dense", _plane(I, "I")[0], _plane(J, "J")[0], _plane(U, "U")[0], _plane(V, "V")[0], H, W, p,
         int(half_win), int(niter), a.ctypes.data, sp, ep, stream_ptr())
    return U, V


# --------------------------------------------------------------------------- A12-A19
def _planes5(t: torch.Tensor, H: int, name: str):
    if t.shape[0] != 5 * H:
        raise ValueError(f"{name}: expected a 5H x W stack")
    return _plane(t, name)


def fb_blur(src: torch.Tensor, half_kernel, planes: int = 1, out=None) -> torch.Tensor:
    hk = np.ascontiguousarray(half_kernel, dtype=np.float32)
    s, HH, W, p = _plane(src, "fb_blur.src")
    out = torch.empty_like(src) if out is None else out
    call("of_fb_blur", s, _plane(out, "fb_blur.out")[0], HH // planes, W, p, planes, hk.ctypes.data, len(hk) - 1,
         stream_ptr())
    return out


def fb_box5(src: torch.Tensor, kh: int, out=None) -> torch.Tensor:
    s, HH, W, p = _plane(src, "fb_box5.src")
    out = torch.empty_like(src) if out is None else out
    call("of_fb_box5", s, _plane(out, "fb_box5.out")[0], HH // 5, W, p, int(kh), stream_ptr())
    return out


def poly_consts(g, xg, xxg, ig, polyN) -> FbPolyConsts:
    c = FbPolyConsts()
    c.polyN = int(polyN)
    for k in range(polyN + 1):
        c.g[k], c.xg[k], c.xxg[k] = float(g[k]), float(xg[k]), float(xxg[k])
    for k in range(4):
        c.ig[k] = float(ig[k])
    return c


def fb_polyexp(src: torch.Tensor, consts: FbPolyConsts, out=None) -> torch.Tensor:
    s, H, W, p = _plane(src, "fb_polyexp.src")
    out = torch.empty((5 * H, W), dtype=torch.float32, device=src.device) if out is None else out
    if out.stride(0) != p:
        raise ValueError("fb_polyexp: out must share the source pitch")
    call("of_fb_polyexp", s, _plane(out, "fb_polyexp.out")[0], H, W, p, ctypes.byref(consts), stream_ptr())
    return out


def fb_polyexp_blurred(src: torch.Tensor, half_kernel, consts: FbPolyConsts, out=None) -> torch.Tensor:
    """fb_polyexp(fb_blur(src, half_kernel, 1)) for a 3-tap blur, in one launch."""
    hk = np.ascontiguousarray(half_kernel, dtype=np.float32)
    if hk.shape != (2,):
        raise ValueError("fb_polyexp_blurred: the blur must have 3 taps (half kernel of 2)")
    s, H, W, p = _plane(src, "fb_polyexp_blurred.src")
    out = torch.empty((5 * H, W), dtype=torch.float32, device=src.device) if out is None else out
    if out.stride(0) != p:
        raise ValueError("fb_polyexp_blurred: out must share the source pitch")
    call("of_fb_polyexp_blurred", s, _plane(out, "fb_polyexp_blurred.out")[0], H, W, p, hk.ctypes.data,
         ctypes.byref(consts), stream_ptr())
    return out


def fb_update_matrices(fx, fy, R0, R1, M=None) -> torch.Tensor:
    H, W = fx.shape
    p = _same_pitch(fx, fy)
    M = torch.empty((5 * H, W), dtype=torch.float32, device=fx.device) if M is None else M
    call("of_fb_update_matrices", _plane(fx, "fx")[0], _plane(fy, "fy")[0], _planes5(R0, H, "R0")[0],
         _planes5(R1, H, "R1")[0], _planes5(M, H, "M")[0], H, W, p, stream_ptr())
    return M


def fb_update_flow(M, H, fx=None, fy=None):
    W = M.shape[1]
    fx = torch.empty((H, W), dtype=torch.float32, device=M.device) if fx is None else fx
    fy = torch.empty((H, W), dtype=torch.float32, device=M.device) if fy is None else fy
    call("of_fb_update_flow", _planes5(M, H, "M")[0], _plane(fx, "fx")[0], _plane(fy, "fy")[0], H, W, fx.stride(0),
         stream_ptr())
    return fx, fy


def fb_iteration(M_in, M_out, R0, R1, fx, fy, half_kernel, update_matrices: bool):
    H, W = fx.shape
    hk = np.ascontiguousarray(half_kernel, dtype=np.float32)
    mo = _planes5(M_out, H, "M_out")[0] if M_out is not None else None
    call("of_fb_iteration", _planes5(M_in, H, "M_in")[0], mo, _planes5(R0, H, "R0")[0], _planes5(R1, H, "R1")[0],
         _plane(fx, "fx")[0], _plane(fy, "fy")[0], H, W, fx.stride(0), hk.ctypes.data, len(hk) - 1,
         int(bool(update_matrices)), stream_ptr())
    return fx, fy
