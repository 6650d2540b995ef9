"""Drop-in for the reference's GaussianKernelBitExact module
(src/GaussianKernelBitExact.py:55-144): OpenCV's bit-exact Gaussian kernel restated with
decimal arithmetic.  Host-side constant generation (a handful of taps per call).

Quirk kept from the reference (:102-106): a positive sigma is ignored and
sigma = 0.15 * n + 0.35 is used; sigma <= 0 with n in {1,3,5,7,9} uses fixed tables.
Returns (sum, kernel) with both as float64, like the reference.
"""
import functools
from decimal import Decimal

import numpy as np

_FIXED = {
    1: [1.0],
    3: [0.25, 0.5, 0.25],
    5: [0.0625, 0.25, 0.375, 0.25, 0.0625],
    7: [0.03125, 0.109375, 0.21875, 0.28125, 0.21875, 0.109375, 0.03125],
    9: [4 / 256, 13 / 256, 30 / 256, 51 / 256, 60 / 256, 51 / 256, 30 / 256, 13 / 256, 4 / 256],
}


def getGaussianKernelBitExact(n, sigma):
    s, k = _bitexact_cached(int(n), float(sigma))
    return s, k.copy()


@functools.lru_cache(maxsize=256)
def _bitexact_cached(n, sigma):
    assert n > 0
    if sigma <= 0 and n in _FIXED:
        k = np.array(_FIXED[n], dtype=np.float64)
        return Decimal("1.0"), k  # the fixed tables are returned with a unit sum
    one = Decimal("1.0")
    sigx = Decimal(sigma) if sigma < 0 else Decimal(n) * Decimal("0.15") + Decimal("0.35")
    scale2 = Decimal("-0.125") / (sigx * sigx)
    half = int((n - 1) / 2)
    vals = []
    x = 1 - n
    s = Decimal("0.0")
    for _ in range(half):
        t = (Decimal(x * x) * scale2).exp()
        vals.append(t)
        s += t
        x += 2
    s *= Decimal(2.0)
    s += one
    if (n & 1) == 0:
        s += one
    mul = one / s
    res = [Decimal(0)] * n
    s2 = Decimal("0.0")
    for i in range(half):
        t = vals[i] * mul
        res[i] = t
        res[n - 1 - i] = t
        s2 += t
    s2 *= Decimal(2.0)
    res[half] = one * mul
    s2 += res[half]
    if (n & 1) == 0:
        res[half + 1] = res[half]
        s2 += res[half]
    return np.float64(s2), np.array([float(v) for v in res], dtype=np.float64)
