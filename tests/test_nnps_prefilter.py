"""The FP32 prefilter of the neighbour search decides exactly as FP64 does.

k_nnps first tests each candidate pair in FP32 on coordinates relative to the
grid minimum and only falls back to the FP64 test of partisearching
(CPP_3-NNPS.cpp:300-312: sqrt of the FP64 sum of squares <= h_i + h_j) when the
FP32 squared distance lies within a rounding margin M of T^2.  This file
restates that prefilter in numpy float32 arithmetic, operation for
operation (fused multiply-adds emulated), and checks on adversarial pairs (distances within a few ulps of the
support radius, far from the grid origin) that every pair it decides without
the fallback is decided as the FP64 test decides it.
"""
import numpy as np

U = np.float32(5.9604645e-8)      # 2^-24


def fp64_inside(xi, xj, hi, hj):
    d2 = np.zeros(len(xi))
    for k in range(xi.shape[1]):
        d2 = d2 + (xi[:, k] - xj[:, k]) * (xi[:, k] - xj[:, k])
    T = 2 * ((hi + hj) / 2)
    return np.sqrt(d2) <= T


def _fma32(a, b, c):
    """float32 fused multiply-add: the product of two float32 values is exact
    in float64, so one float64 sum rounded to float32 (a double rounding that
    differs from the single rounding only on exact ties) stands in for it."""
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def _bounds(nd, fh, hj, ce, ct):
    f32 = np.float32
    Tf = (fh + hj).astype(f32)
    T2f = (Tf * Tf).astype(f32)
    e = (ce + (f32(4.4) * U * Tf).astype(f32)).astype(f32)
    M = (f32(nd) * e * (f32(4.0) * Tf + e).astype(f32) + (ct * T2f).astype(f32)).astype(f32)
    return (T2f - M).astype(f32), (T2f + M).astype(f32), T2f


def prefilter(xi, xj, hi, hj, xmin):
    """(decided, inside) of the FP32 stage of k_nnps for each pair: the squared
    distance summed with fused multiply-adds; a candidate with the particle's
    own h is decided by the bounds alone, any other is first tested against
    twice the radius."""
    f32 = np.float32
    nd = xi.shape[1]
    fi = (xi - xmin).astype(f32)
    fj = (xj - xmin).astype(f32)
    fh, fjh = hi.astype(f32), hj.astype(f32)
    Fi = np.max(np.abs(fi), axis=1).astype(f32)
    fast = fh > f32(64.0) * U * Fi
    ce = f32(2.2) * U * Fi
    ct = f32(32.0) * U
    t = (fi[:, 0] - fj[:, 0]).astype(f32)
    d2f = (t * t).astype(f32)
    for k in range(1, nd):
        t = (fi[:, k] - fj[:, k]).astype(f32)
        d2f = _fma32(t, t, d2f)
    lo0, hi0, _ = _bounds(nd, fh, fh, ce, ct)
    lo1, hi1, T2f = _bounds(nd, fh, fjh, ce, ct)
    same = fjh == fh
    lo = np.where(same, lo0, lo1)
    hi = np.where(same, hi0, hi1)
    far = ~same & (d2f > f32(4.0) * T2f)
    inside = ~far & (d2f < lo)
    out = far | (d2f > hi)
    decided = fast & (inside | out)
    return decided, fast & inside


def _pairs_near_radius(rng, n, nd, origin_scale, h, rel):
    """Pairs at distance T (1 + rel * r) from points up to origin_scale from the grid minimum."""
    xmin = rng.uniform(-3.0, 3.0, nd)
    xi = xmin + rng.uniform(0.0, origin_scale, (n, nd))
    d = rng.standard_normal((n, nd))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    hi = np.full(n, h) * (1.0 + 0.1 * rng.integers(0, 2, n))
    hj = np.full(n, h)
    T = hi + hj
    dist = T * (1.0 + rel * rng.uniform(-1.0, 1.0, n))
    xj = xi + d * dist[:, None]
    return xi, xj, hi, hj, xmin


def test_prefilter_agrees_with_fp64_near_the_radius():
    rng = np.random.default_rng(20261203)
    total_decided = 0
    for nd in (2, 3):
        for scale, h in ((1.0, 0.005), (20.0, 0.05), (10.0, 0.04), (300.0, 0.01)):
            for rel in (1e-2, 1e-4, 1e-6, 1e-9, 0.0):
                xi, xj, hi, hj, xmin = _pairs_near_radius(rng, 20000, nd, scale, h, rel)
                dec, ins = prefilter(xi, xj, hi, hj, xmin)
                ref = fp64_inside(xi, xj, hi, hj)
                assert np.array_equal(ins[dec], ref[dec]), (nd, scale, h, rel)
                total_decided += int(dec.sum())
    assert total_decided > 0


def test_prefilter_on_lattice_knife_edges():
    """Lattice pairs at exactly 2 h (the reference's knife edge) go to FP64."""
    dx = 0.005
    g = np.arange(-3, 4) * dx
    off = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
    base = np.array([0.4175, 0.2325, 0.1525])
    xi = np.repeat(base[None, :], len(off), axis=0)
    xj = xi + off
    h = np.full(len(off), dx)
    dec, ins = prefilter(xi, xj, h, h, np.zeros(3))
    ref = fp64_inside(xi, xj, h, h)
    assert np.array_equal(ins[dec], ref[dec])
    knife = np.isclose(np.linalg.norm(off, axis=1), 2 * dx, rtol=0, atol=1e-15)
    assert knife.any() and not dec[knife].any()
    assert dec.mean() > 0.8


def test_prefilter_disabled_far_from_origin():
    """h below 64 u |coordinate| sends every candidate to the FP64 test."""
    rng = np.random.default_rng(7)
    xi, xj, hi, hj, xmin = _pairs_near_radius(rng, 1000, 3, 1.0e6, 1.0e-3, 1e-3)
    dec, _ = prefilter(xi, xj, hi, hj, xmin)
    assert not dec.any()
