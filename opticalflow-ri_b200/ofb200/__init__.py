"""ofb200: B200-native (sm_100a) kernels of OpticalFlow-RI's dense pyramidal optical-flow
hot path, behind the reference's Python module / class API.

The drop-in modules sit next to this package (``GenericPyramidalOpticalFlow``,
``HornSchunck``, ``PhysicsBasedOpticalFlowLiuShen``, ``denseLucasKanade_PyCL``,
``Farneback_PyCL``, ``gaussian_filter``, ``GaussianKernelBitExact``); put the directory
that holds them on ``sys.path`` exactly as the reference's examples do with its ``src``.

Inputs may be numpy arrays (copied to the device, results copied back as new numpy
arrays) or CUDA tensors (used in place, results returned as tensors).
"""
from __future__ import annotations

import os

import numpy as np

__version__ = "0.1.0"

VERBOSE = os.environ.get("OFB200_VERBOSE", "0") not in ("", "0")


def log(*args):
    if VERBOSE:
        print(*args)


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("ofb200 needs a CUDA device (B200, sm_100a); there is no CPU fallback")
    return torch


def device_of(platformID=0, deviceID=0):
    """The reference selects an OpenCL platform/device; here deviceID is the CUDA index."""
    torch = _torch()
    n = torch.cuda.device_count()
    if deviceID < 0 or deviceID >= n:
        raise ValueError(f"deviceID {deviceID} out of range (0..{n - 1})")
    return torch.device("cuda", int(deviceID))


def to_device(a, device=None):
    """float32 CUDA plane from a numpy array or tensor (uint8 frames are cast like the
    reference examples' astype(np.float32))."""
    torch = _torch()
    if isinstance(a, torch.Tensor):
        t = a if a.is_cuda else a.to(device or torch.device("cuda", torch.cuda.current_device()))
        if t.dtype != torch.float32:
            t = t.float()
        if t.dim() != 2 or t.stride(1) != 1:
            t = t.contiguous()
        return t
    arr = np.ascontiguousarray(a)
    if arr.ndim != 2:
        raise ValueError("expected a 2-D image")
    if arr.dtype != np.float32:
        arr = arr.astype(np.float32)
    dev = device or torch.device("cuda", torch.cuda.current_device())
    return torch.from_numpy(arr).to(dev, non_blocking=False)


def is_host(a) -> bool:
    return isinstance(a, np.ndarray)


def to_host(t):
    return t.detach().cpu().numpy()


_PINNED_OUT = {}


def par_copyto(dst: np.ndarray, src: np.ndarray) -> None:
    """np.copyto(dst, src) for the staging copies of host-buffer calls.  Same-dtype
    C-contiguous planes go through of_host_copy, which splits a large copy over a small
    pool of native threads (ctypes releases the interpreter lock for the call); anything
    else (a cast, a strided view) through numpy."""
    if (dst.dtype == src.dtype and dst.shape == src.shape and dst.flags.c_contiguous and src.flags.c_contiguous
            and dst.nbytes >= (1 << 20)):
        from ._lib import call
        call("of_host_copy", dst.ctypes.data, src.ctypes.data, dst.nbytes)
        return
    np.copyto(dst, src)


def to_host_pair(a, b):
    """Two same-shape float32 CUDA planes -> two new numpy arrays: asynchronous copies into
    cached pinned buffers; the first plane leaves the pinned buffer (threaded host copy)
    while the second is still being downloaded."""
    torch = _torch()
    key = (tuple(a.shape), a.device.index)
    if a.shape != b.shape or a.dtype != torch.float32 or b.dtype != torch.float32:
        return to_host(a), to_host(b)
    buf = _PINNED_OUT.get(key)
    if buf is None:
        buf = _PINNED_OUT[key] = (torch.empty(a.shape, dtype=torch.float32, pin_memory=True),
                                  torch.empty(a.shape, dtype=torch.float32, pin_memory=True), torch.cuda.Event())
    stream = torch.cuda.current_stream(a.device)
    buf[0].copy_(a, non_blocking=True)
    buf[2].record(stream)
    buf[1].copy_(b, non_blocking=True)
    out = (np.empty(a.shape, dtype=np.float32), np.empty(b.shape, dtype=np.float32))
    buf[2].synchronize()
    par_copyto(out[0], buf[0].numpy())
    stream.synchronize()
    par_copyto(out[1], buf[1].numpy())
    return out
