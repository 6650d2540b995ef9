"""The Horn-Schunck sweeps divide num / den as RN32(RN64(num * RN64(1 / den))) (hq_div in
csrc/hsweep.cuh: the reciprocal of each cell's denominator is computed once, so a sweep's
rows carry no division branch).  The claim is that this is the correctly rounded float32
quotient for all float32 operands.  Checked here with numpy's IEEE float32 division as the
answer: random bit patterns (subnormals, infinities, NaNs included), the denominators the
solver forms (alpha^2 + fx^2 + fy^2), denominators with all-ones significands, and
numerators built to put the quotient next to a rounding midpoint."""
import numpy as np


def _div_via_recip(num, den):
    rd = np.float64(1.0) / den.astype(np.float64)
    with np.errstate(invalid="ignore", over="ignore"):
        return (num.astype(np.float64) * rd).astype(np.float32)


def _check(num, den):
    with np.errstate(divide="ignore", invalid="ignore", over="ignore", under="ignore"):
        want = num / den
        got = _div_via_recip(num, den)
    bad = ~(np.isnan(want) & np.isnan(got)) & (want.view(np.uint32) != got.view(np.uint32))
    assert not bad.any(), (num[bad][:4], den[bad][:4], want[bad][:4], got[bad][:4])


def test_random_bit_patterns():
    rng = np.random.default_rng(1)
    for _ in range(8):
        num = rng.integers(0, 2**32, size=1 << 21, dtype=np.uint64).astype(np.uint32).view(np.float32)
        den = rng.integers(0, 2**32, size=1 << 21, dtype=np.uint64).astype(np.uint32).view(np.float32)
        _check(num, den)


def test_special_values():
    sp = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1.0, -1.0, 1e-45, -1e-45, 1.1754942e-38, 3.4028235e38,
                   -3.4028235e38, 5.877472e-39, 2.0 ** -126, 2.0 ** 127], dtype=np.float32)
    num, den = np.meshgrid(sp, sp)
    _check(num.ravel(), den.ravel())


def test_solver_denominators():
    """den = (a2 + fx*fx) + fy*fy in float32 as the sweep forms it, with numerators of the
    solver's range."""
    rng = np.random.default_rng(2)
    n = 1 << 22
    for a2 in (np.float32(441.0), np.float32(1.0), np.float32(0.25), np.float32(1e-6)):
        fx = (rng.standard_normal(n) * rng.choice([1e-3, 1.0, 30.0, 1e3], n)).astype(np.float32)
        fy = (rng.standard_normal(n) * rng.choice([1e-3, 1.0, 30.0, 1e3], n)).astype(np.float32)
        den = (a2 + fx * fx) + fy * fy
        num = (rng.standard_normal(n) * rng.choice([1e-6, 1e-2, 1.0, 1e2, 1e5], n)).astype(np.float32)
        _check(num, den)


def test_all_ones_significands_and_near_midpoints():
    rng = np.random.default_rng(3)
    n = 1 << 20
    # denominators 1.111...1 x 2^e and random ones
    e = rng.integers(-120, 120, n)
    den_ones = np.ldexp(np.float64(2 ** 24 - 1) / 2 ** 23, e).astype(np.float32)
    den_rand = rng.uniform(1.0, 2.0, n).astype(np.float32) * np.ldexp(np.float32(1.0), rng.integers(-60, 60, n)).astype(np.float32)
    for den in (den_ones, den_rand):
        # a float32 quotient q and its midpoint with the next float; numerators rounding den * mid
        q = rng.uniform(1.0, 2.0, n).astype(np.float32) * np.ldexp(np.float32(1.0), rng.integers(-40, 40, n)).astype(np.float32)
        mid = (q.astype(np.float64) + np.nextafter(q, np.float32(np.inf)).astype(np.float64)) / 2
        with np.errstate(over="ignore"):
            base = (den.astype(np.float64) * mid).astype(np.float32)
        for k in range(-3, 4):
            num = base.view(np.int32) + np.int32(k)
            num = num.view(np.float32)
            ok = np.isfinite(num)
            _check(num[ok], den[ok])


def test_subnormal_quotients():
    rng = np.random.default_rng(4)
    n = 1 << 21
    num = rng.uniform(-1, 1, n).astype(np.float32) * np.float32(2.0 ** -100)
    den = rng.uniform(1, 2, n).astype(np.float32) * np.ldexp(np.float32(1.0), rng.integers(20, 60, n)).astype(np.float32)
    _check(num, den)
    assert np.any(np.abs(num / den) < np.float32(2.0 ** -126))  # the subnormal range is exercised
