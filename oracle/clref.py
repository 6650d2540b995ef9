"""The reference's OpenCL kernels run on the host CPU (TEST INFRASTRUCTURE ONLY).

``oracle/clref/`` compiles the reference's own kernel files (src/optical_flow_farneback.cl,
src/pyrlkDenseLargeW.cl) into host libraries under ``oracle/_ref/`` (see its Makefile and
clshim.hpp: an OpenCL-C-to-C++ shim, a fiber executor for work-groups and barriers, and
an exact-float32 bilinear sampler in place of the device's fixed-point texture filter).
This module loads them and offers two ways in:

* kernel-level calls with the reference host's launch geometry (``polyexp``, ``blur``,
  ``blur5``, ``box5``, ``update_matrices``, ``update_flow``, ``lk_dense``), for tests that
  compare the C restatement (of_oracle.c) with the reference's kernels directly;
* ``fake_pyopencl()``: stand-in ``pyopencl`` modules whose Program/Kernel/Buffer objects
  run those libraries, so the reference's unmodified host modules (Farneback_PyCL.py,
  denseLucasKanade_PyCL.py) and its pyramid driver can be executed here to make golden
  vectors (tests/golden/make_golden_cl.py).

Only tests/ and the golden scripts use this module.  Each library exists in two builds:
``fma`` (floating-point contraction, as OpenCL compilers do by default) and ``nofma``.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import re
import subprocess
import types

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
_libs: dict = {}

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
I, Z, P = ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p


def build(reference_src: str) -> None:
    """Compile the libraries from the reference's src/ directory."""
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(_HERE, "clref"), f"REFERENCE_SRC={reference_src}"],
                   check=True)


def available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libclref_fb_polyN7_fma.so"))


def lib(name: str, contract: bool = True):
    """name: 'fb_polyN5', 'fb_polyN7', 'lk_ws1', 'lk_ws0'."""
    key = (name, contract)
    if key not in _libs:
        path = os.path.join(REF_DIR, f"libclref_{name}_{'fma' if contract else 'nofma'}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle/clref REFERENCE_SRC=<reference>/src)")
        L = ctypes.CDLL(path)
        if name.startswith("fb"):
            L.clref_polynomialExpansion.argtypes = [P, I, P, I, I, I, P, P, P, Z, P, Z, Z, Z, Z]
            L.clref_gaussianBlur.argtypes = [P, I, P, I, I, I, P, I, Z, Z, Z, Z, Z]
            L.clref_gaussianBlur5.argtypes = [P, I, P, I, I, I, P, I, Z, Z, Z, Z, Z]
            L.clref_boxFilter5.argtypes = [P, I, P, I, I, I, I, Z, Z, Z, Z, Z]
            L.clref_updateMatrices.argtypes = [P, I, P, I, I, I, P, I, P, I, P, I, Z, Z, Z, Z]
            L.clref_updateFlow.argtypes = [P, I, P, I, P, I, I, I, Z, Z, Z, Z]
        else:
            L.clref_lkDense.argtypes = [P, P, I, I, P, P, P, P] + [I] * 13 + [Z, Z, Z, Z]
        _libs[key] = L
    return _libs[key]


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"clref {what}: work-items diverged on a barrier (rc {rc})")


# ---- kernel-level calls with the reference host's launch geometry --------------------------
def polyexp(src, polyN, g, xg, xxg, ig, contract=True):
    """Farneback_PyCL.polynomialExpansion (src/Farneback_PyCL.py:310-352)."""
    src = np.ascontiguousarray(src, np.float32)
    H, W = src.shape
    dst = np.zeros((5 * H, W), np.float32)
    g, xg, xxg = (np.ascontiguousarray(t, np.float32) for t in (g, xg, xxg))
    ig = np.ascontiguousarray(ig, np.float32)
    wg = 256
    g0 = (W + wg - 2 * polyN - 1) // (wg - 2 * polyN) * wg
    _check(lib(f"fb_polyN{polyN}", contract).clref_polynomialExpansion(
        _ptr(src), W, _ptr(dst), W, H, W, _ptr(g), _ptr(xg), _ptr(xxg), 3 * wg * 4, _ptr(ig), g0, H, wg, 1), "polyexp")
    return dst


def blur(src, half_kernel, ksize_half, contract=True, polyN=7):
    """Farneback_PyCL.gaussianBlur (src/Farneback_PyCL.py:209-238)."""
    src = np.ascontiguousarray(src, np.float32)
    H, W = src.shape
    dst = np.zeros_like(src)
    k = np.ascontiguousarray(half_kernel, np.float32)
    _check(lib(f"fb_polyN{polyN}", contract).clref_gaussianBlur(
        _ptr(src), W, _ptr(dst), W, H, W, _ptr(k), int(ksize_half), (256 + 2 * int(ksize_half)) * 4, W, H, 256, 1),
        "gaussianBlur")
    return dst


def blur5(src5, half_kernel, ksize_half, contract=True, polyN=7):
    """Farneback_PyCL.gaussianBlur5 (src/Farneback_PyCL.py:240-270)."""
    src5 = np.ascontiguousarray(src5, np.float32)
    H5, W = src5.shape
    dst = np.zeros_like(src5)
    k = np.ascontiguousarray(half_kernel, np.float32)
    kh = int(ksize_half)
    _check(lib(f"fb_polyN{polyN}", contract).clref_gaussianBlur5(
        _ptr(src5), W, _ptr(dst), W, H5 // 5, W, _ptr(k), kh, (256 + 2 * kh) * 5 * 4, W, H5 // 5, 256, 1),
        "gaussianBlur5")
    return dst


def box5(src5, ksize_half, contract=True, polyN=7):
    """Farneback_PyCL.boxFilter5 (src/Farneback_PyCL.py:272-308)."""
    src5 = np.ascontiguousarray(src5, np.float32)
    H5, W = src5.shape
    dst = np.zeros_like(src5)
    kh = int(ksize_half)
    _check(lib(f"fb_polyN{polyN}", contract).clref_boxFilter5(
        _ptr(src5), W, _ptr(dst), W, H5 // 5, W, kh, (256 + 2 * kh) * 5 * 4, W, H5 // 5, 256, 1), "boxFilter5")
    return dst


def update_matrices(fx, fy, RA, RB, contract=True, polyN=7):
    """Farneback_PyCL.updateMatrices (src/Farneback_PyCL.py:384-415)."""
    fx, fy, RA, RB = (np.ascontiguousarray(t, np.float32) for t in (fx, fy, RA, RB))
    H, W = fx.shape
    M = np.zeros((5 * H, W), np.float32)
    _check(lib(f"fb_polyN{polyN}", contract).clref_updateMatrices(
        _ptr(fx), W, _ptr(fy), W, H, W, _ptr(RA), W, _ptr(RB), W, _ptr(M), W, W, H, 32, 8), "updateMatrices")
    return M


def update_flow(M, contract=True, polyN=7):
    """Farneback_PyCL.updateFlow (src/Farneback_PyCL.py:354-382)."""
    M = np.ascontiguousarray(M, np.float32)
    H5, W = M.shape
    H = H5 // 5
    fx, fy = np.zeros((H, W), np.float32), np.zeros((H, W), np.float32)
    _check(lib(f"fb_polyN{polyN}", contract).clref_updateFlow(
        _ptr(M), W, _ptr(fx), W, _ptr(fy), W, H, W, W, H, 32, 8), "updateFlow")
    return fx, fy


def lk_dense(I_, J_, U, V, half_win=13, niter=5, asym=(0, 0, 0, 0), contract=True):
    """denseLucasKanade_PyCl.compute's launch of lkDense (src/denseLucasKanade_PyCL.py:113-169):
    level 0, calcErr 1, one 8x8 work-group per pixel.  Returns U, V, status, err (status
    and err in buffers of the right width, unlike the reference's host)."""
    I_, J_ = np.ascontiguousarray(I_, np.float32), np.ascontiguousarray(J_, np.float32)
    H, W = I_.shape
    u = np.ascontiguousarray(U, np.float32).ravel().copy()
    v = np.ascontiguousarray(V, np.float32).ravel().copy()
    status = np.ones(H * W, np.uint8)
    err = np.zeros(H * W, np.float32)
    ws = 2 * half_win + 1
    name = "lk_ws1" if ws >= 16 else "lk_ws0"
    bx, by = (32, 8) if ws > 32 and ws > 2 * ws else (16, 16)
    px, py = (ws + bx - 1) // bx, (ws + by - 1) // by
    _check(lib(name, contract).clref_lkDense(
        _ptr(I_), _ptr(J_), H, W, _ptr(u), _ptr(v), _ptr(status), _ptr(err), 0, H, W, px, py, ws, ws,
        int(asym[0]), int(asym[1]), int(asym[2]), int(asym[3]), int(niter), 1, 8 * H * W, 8, 8, 8), "lkDense")
    return u.reshape(H, W), v.reshape(H, W), status.reshape(H, W), err.reshape(H, W)


# ---- stand-in pyopencl ------------------------------------------------------------------
def _source_hashes():
    out = {}
    path = os.path.join(REF_DIR, "sources.sha256")
    if os.path.exists(path):
        for line in open(path):
            h, name = line.split()
            out[h] = name
    return out


def fake_pyopencl(contract: bool = True):
    """Modules {'pyopencl', 'pyopencl.array', 'pyopencl.cltypes'} that run the reference's
    host code on the clref libraries.  Program(ctx, src).build(options) accepts only the
    exact kernel file that was compiled (checked by SHA-256) and picks the library from the
    -DpolyN / -DWSX options.  Buffers carry 4x slack so the reference's lkDense `err`
    writes (float32 stores into a uint8 buffer) stay inside the allocation."""
    cl = types.ModuleType("pyopencl")
    cla = types.ModuleType("pyopencl.array")
    clt = types.ModuleType("pyopencl.cltypes")
    clt.int, clt.char, clt.float, clt.uint8, clt.uint = np.int32, np.int8, np.float32, np.uint8, np.uint32
    vec = types.SimpleNamespace(float4=np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("w", "<f4")]),
                                double4=np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("w", "<f8")]))
    cla.vec = vec
    cl.array = cla
    cl.cltypes = clt
    cl.mem_flags = types.SimpleNamespace(READ_ONLY=1, WRITE_ONLY=2, READ_WRITE=4, COPY_HOST_PTR=8,
                                         ALLOC_HOST_PTR=16, USE_HOST_PTR=32)
    cl.device_info = types.SimpleNamespace(IMAGE_SUPPORT="IMAGE_SUPPORT")
    hashes = _source_hashes()

    class Device:
        def get_info(self, what):
            return True

        def __str__(self):
            return "<host CPU running the reference's OpenCL kernels (clref)>"

    class Platform:
        def get_devices(self):
            return [Device()]

    cl.get_platforms = lambda: [Platform()]
    cl.Context = lambda devs: types.SimpleNamespace(devices=devs)
    cl.CommandQueue = lambda ctx: types.SimpleNamespace(ctx=ctx)

    class Buffer:
        def __init__(self, ctx, flags, size=None, hostbuf=None):
            n = hostbuf.nbytes if hostbuf is not None else int(size)
            self.nbytes = n
            self.data = np.zeros(4 * n + 64, np.uint8)
            if hostbuf is not None:
                self.data[:n] = np.frombuffer(np.ascontiguousarray(hostbuf).tobytes(), np.uint8)

    class LocalMemory:
        def __init__(self, size):
            self.size = int(size)

    class Image:
        def __init__(self, arr):
            self.arr = np.ascontiguousarray(arr, np.float32)

    def image_from_array(ctx, arr, num_channels=1, mode="r"):
        assert num_channels == 1 and arr.ndim == 2
        return Image(arr)

    def enqueue_copy(queue, dst, src):
        assert isinstance(src, Buffer) and isinstance(dst, np.ndarray)
        flat = dst.reshape(-1).view(np.uint8)
        flat[:] = src.data[:dst.nbytes]

    cl.Buffer, cl.LocalMemory, cl.image_from_array, cl.enqueue_copy = Buffer, LocalMemory, image_from_array, enqueue_copy

    def arg(a):
        if isinstance(a, Buffer):
            return a.data.ctypes.data
        if isinstance(a, Image):
            return a
        if isinstance(a, LocalMemory):
            return a.size
        if isinstance(a, np.ndarray) and a.dtype.names:  # float4 by value
            return np.array([a[n][0] for n in ("x", "y", "z", "w")], np.float32)
        return int(a)

    class Kernel:
        def __init__(self, L, name):
            self.L, self.name = L, name

        def __call__(self, queue, gsize, lsize, *args):
            a = [arg(x) for x in args]
            g0, g1 = int(gsize[0]), int(gsize[1])
            l0, l1 = int(lsize[0]), int(lsize[1])
            n = self.name
            if n == "polynomialExpansion":
                ig = a[10]
                rc = self.L.clref_polynomialExpansion(*a[:9], a[9], ig.ctypes.data, g0, g1, l0, l1)
            elif n in ("gaussianBlur", "gaussianBlur5"):
                rc = getattr(self.L, "clref_" + n)(*a[:9], g0, g1, l0, l1)
            elif n == "boxFilter5":
                rc = self.L.clref_boxFilter5(*a[:8], g0, g1, l0, l1)
            elif n == "updateMatrices":
                rc = self.L.clref_updateMatrices(*a[:12], g0, g1, l0, l1)
            elif n == "updateFlow":
                rc = self.L.clref_updateFlow(*a[:8], g0, g1, l0, l1)
            elif n == "lkDense":
                im1, im2 = a[0], a[1]
                assert im1.arr.shape == im2.arr.shape
                H, W = im1.arr.shape
                rc = self.L.clref_lkDense(im1.arr.ctypes.data, im2.arr.ctypes.data, H, W, *a[2:19], g0, g1, l0, l1)
            else:
                raise NotImplementedError(n)
            _check(rc, n)

    class Program:
        def __init__(self, ctx, src):
            h = hashlib.sha256(src.encode()).hexdigest()
            if h not in hashes:
                raise RuntimeError("clref: the kernel source given to Program() is not the file that was compiled")
            self.file = hashes[h]

        def build(self, options=()):
            opts = " ".join(options)
            if self.file.startswith("optical_flow_farneback"):
                if "-DUSE_DOUBLE" in opts:
                    raise NotImplementedError("clref: the USE_DOUBLE build is not compiled")
                m = re.search(r"-DpolyN=(\d+)", opts)
                L = lib(f"fb_polyN{m.group(1) if m else 5}", contract)
                names = ("polynomialExpansion", "gaussianBlur", "gaussianBlur5", "updateMatrices", "boxFilter5",
                         "updateFlow")
            else:
                mx, my = re.search(r"-DWSX=(\d)", opts), re.search(r"-DWSY=(\d)", opts)
                wsx, wsy = (mx.group(1) if mx else "0"), (my.group(1) if my else "0")
                if wsx != wsy:
                    raise NotImplementedError("clref: only WSX == WSY builds are compiled")
                L = lib(f"lk_ws{wsx}", contract)
                names = ("lkDense",)
            for nm in names:
                setattr(self, nm, Kernel(L, nm))
            return self

    cl.Program = Program
    return {"pyopencl": cl, "pyopencl.array": cla, "pyopencl.cltypes": clt}
