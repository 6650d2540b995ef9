"""ctypes binding of libofb200.so (the sm_100a kernels behind include/ofb200.h).

The library is built in-tree by ``opticalflow-ri_b200/csrc/Makefile``.  There is no
fallback: if the library is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libofb200.so")
CSRC = os.path.join(os.path.dirname(_HERE), "csrc")

OF_OK = 0
OF_FILTER_BILINEAR = 0
OF_FILTER_BICUBIC = 1


class OfError(RuntimeError):
    """A C-ABI entry point returned a negative status."""


class OfHsBatchPair(ctypes.Structure):
    _fields_ = [("I0", ctypes.c_void_p), ("I1", ctypes.c_void_p), ("U", ctypes.c_void_p), ("V", ctypes.c_void_p),
                ("H", ctypes.c_int), ("W", ctypes.c_int), ("pitch", ctypes.c_int), ("alpha", ctypes.c_float),
                ("niter", ctypes.c_int)]


class OfTuning(ctypes.Structure):
    _fields_ = [("tile_shape", ctypes.c_int), ("streams", ctypes.c_int), ("hs_arithmetic", ctypes.c_int),
                ("hs_schedule", ctypes.c_int)]


# per-pair status bits (include/ofb200.h)
ST_NONFINITE_INPUT, ST_WAIT_TIMEOUT, ST_NOT_CONVERGED, ST_SINGULAR, ST_NONFINITE_OUTPUT = 0x1, 0x2, 0x4, 0x8, 0x10


class FbPolyConsts(ctypes.Structure):
    _fields_ = [("polyN", ctypes.c_int), ("g", ctypes.c_float * 8), ("xg", ctypes.c_float * 8),
                ("xxg", ctypes.c_float * 8), ("ig", ctypes.c_float * 4)]


OF_FB_MAX_LEVELS = 8
OF_METHOD_HS, OF_METHOD_LK, OF_METHOD_FB = 0, 1, 2


class OfFbParams(ctypes.Structure):
    _fields_ = [("window_size", ctypes.c_int), ("niters", ctypes.c_int), ("use_gaussian", ctypes.c_int),
                ("levels", ctypes.c_int), ("pyr_scale", ctypes.c_double), ("poly", FbPolyConsts),
                ("window_taps", ctypes.c_void_p), ("window_kh", ctypes.c_int),
                ("level_taps", ctypes.c_void_p * OF_FB_MAX_LEVELS), ("level_kh", ctypes.c_int * OF_FB_MAX_LEVELS)]


class OfPairDesc(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int), ("frame_u8", ctypes.c_int), ("I0", ctypes.c_void_p),
                ("I1", ctypes.c_void_p), ("in_pitch", ctypes.c_int), ("U", ctypes.c_void_p), ("V", ctypes.c_void_p),
                ("out_pitch", ctypes.c_int), ("H", ctypes.c_int), ("W", ctypes.c_int), ("filter", ctypes.c_float),
                ("filter_taps", ctypes.c_void_p), ("levels", ctypes.c_int), ("refine_ls", ctypes.c_int),
                ("filter_opt", ctypes.c_float), ("filter_opt_taps", ctypes.c_void_p), ("ls_h", ctypes.c_float),
                ("ls_arithmetic", ctypes.c_int), ("warping", ctypes.c_int), ("intermediate_scaling", ctypes.c_int),
                ("scaling", ctypes.c_int), ("hs_alphas", ctypes.c_float * 8), ("hs_nalphas", ctypes.c_int),
                ("hs_niter", ctypes.c_int), ("lk_half_win", ctypes.c_int), ("lk_niter", ctypes.c_int),
                ("fb", ctypes.c_void_p)]


_lib = None

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_D = ctypes.c_double
_Z = ctypes.c_size_t
_L = ctypes.c_longlong

_SIGS = {
    "of_version": ([], _I),
    "of_last_error": ([ctypes.c_char_p, _Z], _I),
    "of_launch_count": ([], ctypes.c_ulonglong),
    "of_host_copy": ([_P, _P, _Z], _I),
    "of_prefilter_f32": ([_P, _I, _P, _I, _I, _I, _P, _I, _P], _I),
    "of_prefilter_u8": ([_P, _I, _P, _I, _I, _I, _P, _I, _P], _I),
    "of_u8_to_f32": ([_P, _I, _P, _I, _I, _I, _P], _I),
    "of_u16_to_f32": ([_P, _I, _P, _I, _I, _I, _P], _I),
    "of_resize_workspace_size": ([_I, _I, _I, _I, _I], _Z),
    "of_resize": ([_P, _I, _I, _I, _P, _I, _I, _I, _I, _P, _Z, _P], _I),
    "of_resize_table_size": ([_I, _I, _I], _Z),
    "of_resize_table": ([_I, _I, _I, _P, _Z, _P], _I),
    "of_resize_tabled": ([_P, _I, _I, _I, _P, _I, _I, _I, _I, _P, _P, _P, _Z, _P], _I),
    "of_spline_workspace_size": ([_I, _I, _I, _I], _Z),
    "of_spline_upsample": ([_P, _I, _I, _I, _P, _I, _I, _I, _F, _P, _Z, _P], _I),
    "of_spline_upsample_pair": ([_P, _P, _I, _I, _I, _P, _P, _I, _I, _I, _F, _F, _P, _Z, _P], _I),
    "of_warp_pair_bilinear": ([_P, _P, _P, _P, _P, _P, _I, _I, _I, _P], _I),
    "of_warp_bilinear_coords": ([_P, _P, _P, _P, _I, _I, _I, _P], _I),
    "of_accumulate": ([_P, _P, _I, _I, _I, _P], _I),
    "of_scale": ([_P, _P, _F, _I, _I, _I, _P], _I),
    "of_hs_workspace_size": ([_I, _I, _I], _Z),
    "of_hs_derivatives": ([_P, _P, _P, _P, _P, _I, _I, _I, _P], _I),
    "of_ls_coefficients": ([_P, _P, _P, _I, _I, _I, _F, _P], _I),
    "of_hs_solve": ([_P, _P, _P, _P, _I, _I, _I, _F, _I, _P, _P, _Z, _P], _I),
    "of_hs_solve_persistent": ([_P, _P, _P, _P, _I, _I, _I, _F, _I, _P, _P, _Z, _P], _I),
    "of_ls_workspace_size": ([_I, _I, _I, _I], _Z),
    "of_ls_solve": ([_P, _P, _P, _P, _I, _I, _I, _F, _I, _D, _P, _P, _P, _Z, _P], _I),
    "of_ls_solve_noalloc": ([_P, _P, _P, _P, _I, _I, _I, _F, _I, _D, _P, _P, _P], _I),
    "of_ls_solve_mode": ([_P, _P, _P, _P, _I, _I, _I, _F, _I, _D, _I, _P, _P, _P, _Z, _P], _I),
    "of_hs_batch_shape": ([_I, _P, _P, _P], _I),
    "of_hs_batch_schedule": ([_P, _I, _P, _Z, _P, _P], _I),
    "of_batch_workspace_size": ([_P, _I, _P], _Z),
    "of_batch_run": ([_P, _I, _P, _P, _P, _Z, _P], _I),
    "of_check_finite": ([_P, _I, _I, _I, _P, _I, _P], _I),
    "of_ls_status": ([_P, _P, _I, _D, _P, _P], _I),
    "of_hs_batch_workspace_size": ([_P, _I], _Z),
    "of_hs_batch": ([_P, _I, _P, _P, _L, _P, _Z, _P], _I),
    "of_warp_liushen_workspace_size": ([_I, _I], _Z),
    "of_warp_liushen_scatter": ([_P, _P, _P, _P, _P, _P, _I, _I, _I, _P, _P, _Z, _P], _I),
    "of_warp_liushen_ofe": ([_P, _P, _P, _P, _I, _I, _I, _P], _I),
    "of_cnn_conv3x3": ([_P, _I, _I, _I, _I, _I, _I, _P, _I, _P, _I, _P, _I, _I, _I, _P, _P], _I),
    "of_cnn_conv3x3_wgrad_tc": ([_P, _I, _I, _P, _I, _I, _I, _I, _I, _I, _I, _P, _P, _P], _I),
    "of_cnn_conv3x3_wgrad": ([_P, _I, _I, _P, _I, _I, _I, _I, _I, _I, _I, _P, _P], _I),
    "of_cnn_bias_grad": ([_P, _I, _I, _L, _I, _P, _P], _I),
    "of_cnn_pack_pair": ([_P, _P, _I, _I, _I, _P, _P, _I, _P], _I),
    "of_cnn_avgpool2": ([_P, _I, _I, _I, _I, _I, _I, _P, _I, _I, _P], _I),
    "of_cnn_avgpool2_bwd": ([_P, _I, _I, _I, _I, _I, _I, _P, _I, _I, _I, _P], _I),
    "of_cnn_upsample2": ([_P, _I, _I, _I, _I, _I, _I, _P, _I, _I, _P], _I),
    "of_cnn_upsample2_bwd": ([_P, _I, _I, _I, _I, _I, _I, _P, _I, _I, _P], _I),
    "of_cnn_relu_bwd": ([_P, _I, _I, _P, _I, _I, _L, _I, _P], _I),
    "of_cnn_flow_mse": ([_P, _P, _L, _P, _I, _P, _P], _I),
    "of_cnn_adam": ([_P, _P, _P, _P, _L, _F, _F, _F, _F, _I, _P], _I),
    "of_cnn_pack_weights": ([_P, _I, _I, _I, _I, _I, _P, _P], _I),
    "of_cnn_flow_up": ([_P, _I, _I, _I, _P, _P, _I, _F, _P], _I),
    "of_cnn_split_flow": ([_P, _I, _I, _P, _P, _I, _P], _I),
    "of_lk_dense": ([_P, _P, _P, _P, _I, _I, _I, _I, _I, _P, _P, _P, _P], _I),
    "of_fb_blur": ([_P, _P, _I, _I, _I, _I, _P, _I, _P], _I),
    "of_fb_box5": ([_P, _P, _I, _I, _I, _I, _P], _I),
    "of_fb_polyexp": ([_P, _P, _I, _I, _I, ctypes.POINTER(FbPolyConsts), _P], _I),
    "of_fb_polyexp_blurred": ([_P, _P, _I, _I, _I, _P, ctypes.POINTER(FbPolyConsts), _P], _I),
    "of_fb_update_matrices": ([_P, _P, _P, _P, _P, _I, _I, _I, _P], _I),
    "of_fb_update_flow": ([_P, _P, _P, _I, _I, _I, _P], _I),
    "of_fb_iteration": ([_P, _P, _P, _P, _P, _P, _I, _I, _I, _P, _I, _I, _P], _I),
}


def exported_symbols():
    """Names of every entry point the binding declares (the header's ABI)."""
    return sorted(_SIGS)


def lib():
    """Loads libofb200.so (raises if it is absent: there is no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"ofb200: {LIB_PATH} is not built; run `make -C {CSRC}` "
                              "(or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    lib().of_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int, name: str) -> None:
    if rc != OF_OK:
        raise OfError(f"{name} failed (status {rc}): {last_error()}")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args), name)
