"""I/O on either side of the optical-flow path, as the reference's examples do it.

read_frame   examples/*.py: imread(fn).astype(np.float32) of a single-page grayscale TIFF
             (8-bit, or 10/12-bit in a 16-bit container: the Bits08/10/12 sets).  Read with
             Pillow (skimage is not a dependency here); the same pixel values.
read_raw     the frame in its stored integer type, to upload as uint8 / uint16 and convert
             on the GPU (ops.u8_to_f32 takes both): half or a quarter of the float32 bytes.
save_flow    examples/PyHSchunck_Fs3_4.py:35-51: a MATLAB file with
             velocities{u, v, iaWidth, iaHeight, margins{top, left, bottom, right}} and
             parameters{overlapFactor, imageHeight, imageWidth}.
load_flow    reads such a file back as (U, V).
"""
from __future__ import annotations

import numpy as np

__all__ = ["read_frame", "read_raw", "save_flow", "load_flow"]


def read_raw(path):
    """The frame as stored: uint8 or uint16 (float TIFFs as float32)."""
    from PIL import Image
    with Image.open(path) as im:
        if getattr(im, "n_frames", 1) != 1:
            raise ValueError(f"{path}: multi-page TIFF")
        a = np.array(im)
    if a.ndim != 2:
        raise ValueError(f"{path}: expected a single-channel image, got shape {a.shape}")
    if a.dtype == np.int32 and a.min() >= 0 and a.max() <= 65535:  # Pillow's mode 'I' for 16-bit data
        a = a.astype(np.uint16)
    return a


def read_frame(path) -> np.ndarray:
    """imread(path).astype(np.float32)."""
    return read_raw(path).astype(np.float32)


def save_flow(U, V, filename):
    """The reference examples' MATLAB output (velocities + parameters)."""
    import scipy.io
    U = np.asarray(U.cpu() if hasattr(U, "cpu") else U)
    V = np.asarray(V.cpu() if hasattr(V, "cpu") else V)
    margins = {"top": 0, "left": 0, "bottom": 0, "right": 0}
    results = {"u": U, "v": V, "iaWidth": 1, "iaHeight": 1, "margins": margins}
    parameters = {"overlapFactor": 1.0, "imageHeight": np.size(U, 0), "imageWidth": np.size(U, 1)}
    scipy.io.savemat(filename, mdict={"velocities": results, "parameters": parameters})


def load_flow(filename):
    import scipy.io
    m = scipy.io.loadmat(filename)
    v = m["velocities"][0, 0]
    return np.asarray(v["u"], np.float32), np.asarray(v["v"], np.float32)
