"""The division of the tree's centre-of-mass recurrence, bit for bit.

The recurrence (gravity_tree.rs:113-118: com = (com*M + x*m) / (M + m))
divides through a correction from the correctly rounded reciprocal of the
new total mass where the operands lie in [2^-500, 2^501), and through the
IEEE division elsewhere; `phys_debug_divide` runs exactly that division.
Every quotient must equal the host's IEEE division (numpy float64, round to
nearest even), including quotients within a hair of a rounding midpoint.
The recurrence itself is checked against the oracle by the tree tests.
"""
from fractions import Fraction

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fast_path(a, b):
    """Where the library takes the reciprocal form (its range test)."""
    ea = (a.view(np.uint64) >> np.uint64(52)) & np.uint64(0x7FF)
    eb = b.view(np.uint64) >> np.uint64(52)  # sign bit included: b > 0 only
    a_ok = ((ea >= 523) & (ea <= 1523)) | (a.view(np.uint64) == 0)
    b_ok = (eb >= 523) & (eb <= 1523)
    return a_ok & b_ok


def _check(ctx, a, b):
    q = ctx.debug_divide(a, b)
    with np.errstate(all="ignore"):
        want = a / b
    same = (q.view(np.uint64) == want.view(np.uint64)) | (np.isnan(q) & np.isnan(want))
    bad = np.flatnonzero(~same)
    assert bad.size == 0, "first mismatches: " + ", ".join(
        "%r/%r -> %r want %r" % (a[i], b[i], q[i], want[i]) for i in bad[:5])
    return _fast_path(a, b)


def test_random_operands(ctx):
    rng = np.random.default_rng(11)
    n = 1 << 21
    a = rng.uniform(1.0, 2.0, n) * np.exp2(rng.integers(-60, 60, n)) * rng.choice([-1.0, 1.0], n)
    b = rng.uniform(1.0, 2.0, n) * np.exp2(rng.integers(-60, 60, n))
    fast = _check(ctx, a, b)
    assert fast.all()


def test_centre_of_mass_shaped_operands(ctx):
    """Operands as the recurrence forms them: a = c*M + x*m, b = M + m."""
    rng = np.random.default_rng(12)
    n = 1 << 20
    M = rng.uniform(0.0, 1.0, n) * np.exp2(rng.integers(-20, 20, n))
    m = rng.uniform(1e-6, 1.0, n)
    c = rng.normal(0.0, 3.0, n)
    x = rng.normal(0.0, 3.0, n)
    a = c * M + x * m
    b = M + m
    assert _check(ctx, a, b).mean() > 0.999


def test_quotients_next_to_midpoints(ctx):
    """a = RN(b * mid) for mid halfway between two doubles: a / b lies within
    about 2^-53 ulp of the midpoint, the hardest case for the rounding."""
    rng = np.random.default_rng(13)
    n = 20000
    bs = rng.uniform(1.0, 2.0, n)
    # significands near 1 and near 2, and b with an all-ones significand
    bs[: n // 8] = 2.0 - np.ldexp(rng.integers(1, 64, n // 8).astype(np.float64), -52)
    bs[n // 8: n // 4] = 1.0 + np.ldexp(rng.integers(1, 64, n // 8).astype(np.float64), -52)
    qs = rng.uniform(1.0, 2.0, n)
    qs[: n // 8] = 2.0 - np.ldexp(rng.integers(1, 64, n // 8).astype(np.float64), -52)
    a = np.empty(n)
    for i in range(n):
        q = float(qs[i])
        mid = Fraction(q) + Fraction(np.spacing(q)) / 2
        a[i] = float(Fraction(float(bs[i])) * mid)  # correctly rounded
    scale = np.exp2(rng.integers(-30, 30, n))
    a *= scale
    b = bs * np.exp2(rng.integers(-30, 30, n))
    a[::2] = -a[::2]
    assert _check(ctx, a, b).all()


def test_exact_quotients(ctx):
    rng = np.random.default_rng(14)
    n = 100000
    q = rng.integers(1, 1 << 20, n).astype(np.float64) * np.exp2(rng.integers(-40, 40, n))
    b = rng.integers(1, 1 << 30, n).astype(np.float64) * np.exp2(rng.integers(-40, 40, n))
    a = q * b  # exact: at most 50 significant bits
    assert _check(ctx, a, b).all()


def test_fallback_cases(ctx):
    tiny, huge = np.ldexp(1.0, -700), np.ldexp(1.0, 700)
    a = np.array([0.0, -0.0, 1.0, -1.0, 1.0, 1.0, 1.0, 1.0, tiny, huge, 5e-324, 1.0,
                  np.inf, np.nan, 3.0, 0.0, -0.0, 2.0])
    b = np.array([1.0, 1.0, 0.0, 0.0, -2.0, tiny, huge, 5e-324, 3.0, 3.0, 7.0, np.inf,
                  2.0, 2.0, np.nan, -1.0, 0.0, np.ldexp(1.0, 500)])
    fast = _check(ctx, a, b)
    assert fast[0] and fast[-1] and not fast[1:-1].any()
