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
from fractions import Fraction

import numpy as np


def rn(v: Fraction) -> float:
    return float(v)            # Fraction -> float rounds to nearest, ties to even


def div_by_recip(x: float, y: float, yr: float) -> float:
    q = x * yr                 # an IEEE double product, signed zeros included
    r = rn(Fraction(x) - Fraction(q) * Fraction(y))
    if r == 0.0:
        return q
    return rn(Fraction(r) * Fraction(yr) + Fraction(q))


def _check(xs, ys):
    bad = 0
    for x, y in zip(xs, ys):
        x, y = float(x), float(y)
        yr = 1.0 / y
        got = div_by_recip(x, y, yr)
        want = x / y
        if got != want or np.signbit(got) != np.signbit(want):
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
