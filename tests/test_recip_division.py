"""The quotient by a correctly rounded reciprocal that the pair-record pass
uses in place of three of its four divisions per pair (k_pairw): with
yr = RN(1 / y), q = RN(x yr), r = RN(x - q y) (exact, a fused multiply-add),
RN(q + r yr) is RN(x / y) (Markstein's correction: q is within one ulp of
x / y and yr within half an ulp of 1 / y).  The engine returns q itself when
r is zero, which keeps the sign of a zero quotient.

Checked here on the CPU with exact rational arithmetic standing in for the
device's rounded multiply and fused multiply-adds, against IEEE division,
on random operands over many binades and on quotients near rounding ties.
"""
import math
from fractions import Fraction

import numpy as np


def rn(v: Fraction) -> float:
    return float(v)            # Fraction -> float rounds to nearest, ties to even


def _ieee_div(x: float, y: float) -> float:
    if y == 0.0:
        if x == 0.0 or math.isnan(x):
            return math.nan
        return math.copysign(math.inf, x) * math.copysign(1.0, y)
    return x / y


def _fma_residual(x: float, y: float, q: float) -> float:
    """RN(x - q y), with the IEEE results for infinite and NaN operands."""
    if not (math.isfinite(x) and math.isfinite(y) and math.isfinite(q)):
        with np.errstate(all="ignore"):
            return float(np.float64(x) - np.float64(q) * np.float64(y))
    return rn(Fraction(x) - Fraction(q) * Fraction(y))


def div_by_recip(x: float, y: float, yr: float) -> float:
    with np.errstate(all="ignore"):
        q = float(np.float64(x) * np.float64(yr))    # IEEE product, signed zeros and infinities included
    r = _fma_residual(x, y, q)
    if r == 0.0:
        return q
    if not math.isfinite(r):
        return _ieee_div(x, y)
    return rn(Fraction(r) * Fraction(yr) + Fraction(q))


def _same(a: float, b: float) -> bool:
    if math.isnan(a) or math.isnan(b):
        return math.isnan(a) and math.isnan(b)
    return a == b and np.signbit(a) == np.signbit(b)


def _check(xs, ys):
    bad = 0
    for x, y in zip(xs, ys):
        x, y = float(x), float(y)
        yr = _ieee_div(1.0, y)
        if not _same(div_by_recip(x, y, yr), _ieee_div(x, y)):
            bad += 1
    return bad


def test_random_operands():
    rng = np.random.default_rng(7)
    n = 40000
    xs = rng.uniform(-1.0, 1.0, n) * 2.0 ** rng.integers(-40, 40, n)
    ys = rng.uniform(0.5, 1.0, n) * 2.0 ** rng.integers(-40, 40, n)
    assert _check(xs, ys) == 0


def test_sph_like_operands():
    """The operands of the pair records: numerators a1 dx f(s) and divisors
    ra * dst, ra, 6."""
    rng = np.random.default_rng(11)
    n = 40000
    ra = 0.005 * (1.0 + 0.1 * rng.integers(0, 3, n))
    dst = ra * rng.uniform(1e-3, 2.0, n)
    num = rng.standard_normal(n) * 1e6
    assert _check(num, ra * dst) == 0
    assert _check(dst, ra) == 0
    assert _check(num, np.full(n, 6.0)) == 0


def test_near_ties_and_zeros():
    """Quotients within a few ulps of a rounding tie, exact quotients and
    signed zeros."""
    rng = np.random.default_rng(13)
    xs, ys = [], []
    for _ in range(20000):
        y = float(rng.uniform(1.0, 2.0))
        q = float(rng.uniform(1.0, 2.0))
        # x = (q + half an ulp of q) * y rounded: a quotient near a tie
        x = float(Fraction(q) * Fraction(y) + Fraction(np.spacing(q)) / 2 * Fraction(y))
        xs += [x, np.nextafter(x, 0.0), np.nextafter(x, 4.0), q * y]
        ys += [y, y, y, y]
    xs += [0.0, -0.0, 3.0, -3.0]
    ys += [7.0, 7.0, 3.0, 6.0]
    assert _check(xs, ys) == 0


def test_infinities_nans_and_zero_divisors():
    """Operands a diverging run produces (the reference's own 3-D penalty
    contact drives velocities to infinity): inf / y stays inf, NaN stays NaN,
    x / 0 and x / inf are the IEEE results."""
    xs = [math.inf, -math.inf, math.nan, 1.0, -1.0, 0.0, 2.0, -2.0, math.inf]
    ys = [1590.0, 3.0, 2.0, 0.0, 0.0, 0.0, math.inf, math.inf, math.inf]
    assert _check(xs, ys) == 0
