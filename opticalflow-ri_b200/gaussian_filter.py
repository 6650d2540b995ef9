"""Drop-in for the reference's gaussian_filter module (src/gaussian_filter.py).

The separable prefilter runs on the GPU (of_prefilter_f32 / of_prefilter_u8), bit-exact
with the reference.  As in the reference, convolveSeparableFilter, gaussian_filter and
gaussian_filterPx filter `image` IN PLACE and return it (numpy arrays are written back;
CUDA tensors are overwritten on the device).
"""
import numpy as np

from ofb200 import ops, to_device, is_host, _torch

__all__ = ["prepareGaussianKernel", "convolveSeparableFilter", "gaussian_filter", "gaussian_filterPx"]


def prepareGaussianKernel(sigma, kernelSizePx):
    """Taps of src/gaussian_filter.py:47-52: exp(-x^2/2s^2) at x = -K/2 .. K/2-1 (integer
    positions from np.arange(..., dtype=int)), stored in float32, normalised in float32."""
    kernel = np.zeros(kernelSizePx, dtype=np.float32)
    xs = np.arange(-kernelSizePx / 2, kernelSizePx / 2, 1, dtype=int)
    kernel[:] = 1.0 / np.sqrt(2.0 * np.pi * sigma ** 2) * np.exp(-xs ** 2 / (2.0 * sigma ** 2))
    kernel /= np.sum(kernel)
    return kernel


def _reference_errors(K, H, W):
    """The exceptions src/gaussian_filter.py:54-85 raises before filtering anything: the
    line buffer's slice assignment for K == 1 or an even K, then the border copy reading
    image[i, j] for j < K // 2 (columns first, in the row pass)."""
    h = K // 2
    if K == 1 or K % 2 == 0:
        raise ValueError(f"could not broadcast input array from shape ({W},) into shape ({W + K - 1 - 2 * h if h else 0},)")
    if h > W:
        raise IndexError(f"index {W} is out of bounds for axis 1 with size {W}")
    if h > H:  # the reference has filtered the rows in place when the column pass raises
        raise IndexError(f"index {H} is out of bounds for axis 0 with size {H}")


def convolveSeparableFilter(kernel, image):
    """Row pass then column pass with the reference's border (src/gaussian_filter.py:54-85)."""
    kernel = np.ascontiguousarray(kernel, dtype=np.float32)
    _reference_errors(int(kernel.shape[0]), int(image.shape[0]), int(image.shape[1]))
    if is_host(image):
        src = to_device(image)
        out = ops.prefilter(src, kernel)
        image[...] = out.cpu().numpy().astype(image.dtype, copy=False)
        return image
    torch = _torch()
    src = image if image.dtype in (torch.float32, torch.uint8) else image.float()
    out = ops.prefilter(src.contiguous(), kernel)
    image.copy_(out)
    return image


def gaussian_filter(image, sigma, truncate):
    kernelSizePx = 2 * int(truncate * sigma + 0.5) + 1
    return convolveSeparableFilter(prepareGaussianKernel(sigma, kernelSizePx), image)


def gaussian_filterPx(image, sigma, kernelSizePx):
    return convolveSeparableFilter(prepareGaussianKernel(sigma, kernelSizePx), image)
