"""The FP64 slope-ratio division of the step kernels against IEEE division.

The FP64 kernels divide with a hardware reciprocal estimate, one Newton step and a
Markstein correction (ratio(double) in le2d_b200/csrc/le2d_device.cuh).  Its result is
the correctly rounded quotient unless the exact quotient lies within about 2^-92
(relative) of a midpoint between two doubles, and the FP64 step's bit-for-bit parity with
the reference double build rests on it.  le2d_selftest_ratio evaluates it and CUDA's IEEE
division (__ddiv_rn) side by side on the device.

Domain: the kernels divide a = D' + eps by b = D + eps (or eps - D), with D a difference
of doubles, so b is +0 exactly at a tie and otherwise at least 2^-73 in magnitude, and so
is a.  Tested: operands and quotients between 2^-960 and 2^1020 in magnitude.  Near the
underflow range the Markstein residual itself underflows (numerators below ~2^-970 differ
from IEEE division in the last bit); magnitudes of 2^1022 and above belong to states near
overflow.  Neither occurs in the scheme.  For b = +0 the kernels return copysign(inf, a)
where IEEE gives +-inf, or NaN for 0/0: the limiter maps +inf and NaN alike to 2 and -inf
to 0 (the reference's superbee, le2d simple/le_core.c:38, gives
le_max3(0, le_min(1, NaN), le_min(2, NaN)) = 2).
"""
import numpy as np
import pytest

from le2d_b200 import capi

pytestmark = pytest.mark.gpu

EPS = 1e-6


@pytest.fixture(scope="module")
def lib():
    return capi.Lib("d")


def _random_pairs(rng, n, emin, emax):
    """Signed operands with uniform mantissas and exponents in [emin, emax]."""
    def draw():
        m = rng.uniform(1.0, 2.0, n)
        m[rng.random(n) < 0.05] = 1.0  # powers of two
        return np.ldexp(m, rng.integers(emin, emax + 1, n)) * rng.choice([-1.0, 1.0], n)
    return draw(), draw()


def _slope_pairs(rng, n):
    """a = D' + eps, b = D + eps with D, D' near -eps (a few ulps away), near each other,
    and spread over the values field differences take."""
    ulp = np.spacing(EPS)
    d = -EPS + rng.integers(-40, 41, n) * ulp
    d2 = np.where(rng.random(n) < 0.5, -EPS + rng.integers(-40, 41, n) * ulp,
                  rng.standard_normal(n) * 10.0 ** rng.integers(-9, 2, n))
    b = d + EPS
    a = d2 + EPS
    keep = b != 0.0
    return a[keep], b[keep]


def _exact_quotients(rng, n):
    """Pairs whose quotient is a simple value (breakpoints of the limiter, thirds, ...)."""
    b = rng.uniform(-4.0, 4.0, n) * 10.0 ** rng.integers(-12, 6, n)
    q = rng.choice([0.5, 1.0, 2.0, 1.0 / 3.0, 3.0, -1.0, 0.25, 4.0], n)
    return b * q, b


def test_ratio_matches_ieee_division(lib):
    rng = np.random.default_rng(2024)
    parts = [
        _random_pairs(rng, 1_000_000, -60, 60),
        _random_pairs(rng, 200_000, -900, 900),
        _slope_pairs(rng, 400_000),
        _exact_quotients(rng, 100_000),
    ]
    # operand magnitudes at the edges of the supported range
    bb = np.ldexp(rng.uniform(1.0, 2.0, 20_000), rng.choice([-960, -900, -73, 1000, 1020], 20_000))
    aa = bb * rng.uniform(-3.0, 3.0, 20_000)
    parts.append((aa, bb))
    a = np.concatenate([p[0] for p in parts])
    b = np.concatenate([p[1] for p in parts])
    with np.errstate(over="ignore"):
        q = np.abs(a / b)
    ok = (np.isfinite(q) & (q > 2.0 ** -960) & (q < 2.0 ** 1020) & (np.abs(b) >= 2.0 ** -960)
          & (np.abs(b) < 2.0 ** 1021) & (np.abs(a) >= 2.0 ** -960))
    a, b = a[ok], b[ok]
    fast, ieee = lib.selftest_ratio(a, b)
    assert np.array_equal(ieee, a / b)  # the device's IEEE quotient is the host's
    bad = np.flatnonzero(fast != ieee)
    print(f"\n{a.size} operand pairs; differing from IEEE division: {bad.size}")
    assert bad.size == 0, [(a[i], b[i], fast[i], ieee[i]) for i in bad[:8]]


def test_ratio_zero_divisor(lib):
    a = np.array([1.0, -1.0, 0.0, EPS, -EPS, 2.0 ** -73, -(2.0 ** -73), 1e300, -1e300])
    b = np.zeros_like(a)
    fast, ieee = lib.selftest_ratio(a, b)
    want = np.where(np.signbit(a), -np.inf, np.inf)
    assert np.array_equal(fast, want)
    # IEEE: +-inf where a != 0 (the same), NaN for 0/0, whose superbee (2) is that of +inf
    nz = a != 0.0
    assert np.array_equal(ieee[nz], fast[nz]) and np.isnan(ieee[~nz]).all()


def test_ratio_tie_neighbourhood(lib):
    """Every divisor the scheme can form near a tie, b = (D + eps) for D within 64 ulps of
    -eps, against numerators from the same set and from ordinary slopes."""
    ulp = np.spacing(EPS)
    d = -EPS + np.arange(-64, 65) * ulp
    p = d + EPS
    p = p[p != 0.0]
    a = np.concatenate([np.repeat(p, p.size), np.repeat(np.linspace(-3, 3, 61), p.size)])
    b = np.concatenate([np.tile(p, p.size), np.tile(p, 61)])
    fast, ieee = lib.selftest_ratio(a, b)
    assert np.array_equal(fast, ieee)
