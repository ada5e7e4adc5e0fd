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


def _superbee_reference(r):
    """The reference's superbee (simple/le_core.c:31-38) with its comparison macros:
    le_max(0, le_max(le_min(1, 2r), le_min(2, r))), le_min(a, b) = a > b ? b : a and
    le_max(a, b) = a > b ? a : b -- so superbee(NaN) = 2."""
    with np.errstate(invalid="ignore", over="ignore"):
        two = 2.0 * r
        m1 = np.where(1.0 > two, two, 1.0)
        m2 = np.where(2.0 > r, r, 2.0)
        mx = np.where(m1 > m2, m1, m2)
        return np.where(0.0 > mx, 0.0, mx)


def test_limiter_matches_reference_superbee(lib):
    """The FP64 step's limited slope ratio (psi_ratio: the division fused with the limiter,
    which picks 0, 2r, 1, r or 2 from the quotient's high word) against kc times the
    reference's superbee of the IEEE quotient, bit for bit: random and slope-form operand
    pairs, quotients at and next to the breakpoints 0, 0.5, 1 and 2, and ties (b = +0)."""
    rng = np.random.default_rng(77)
    parts = [_random_pairs(rng, 300_000, -40, 40), _slope_pairs(rng, 300_000), _exact_quotients(rng, 100_000)]
    b = np.ldexp(rng.uniform(1.0, 2.0, 4000), rng.integers(-60, 60, 4000))
    for q in (0.5, 1.0, 2.0, 0.25, 4.0):
        for k in (-2, -1, 0, 1, 2):  # the breakpoint and its neighbours a few ulps away
            qq = q + k * np.spacing(q)
            parts.append((b * qq, b))
    parts.append((-b, b))
    a = np.concatenate([p[0] for p in parts])
    b = np.concatenate([p[1] for p in parts])
    with np.errstate(over="ignore", under="ignore"):
        q = np.abs(a / b)
    ok = (np.isfinite(q) & ((q > 2.0 ** -900) | (q == 0.0)) & (q < 2.0 ** 1000) & (np.abs(b) >= 2.0 ** -900)
          & (np.abs(a) < 2.0 ** 1000))
    a, b = a[ok], b[ok]
    ties = np.array([1.0, -1.0, 0.0, EPS, -EPS, 2.0 ** -73, -(2.0 ** -73), 3.0])
    a = np.concatenate([a, ties])
    b = np.concatenate([b, np.zeros_like(ties)])
    for kc in (0.375, 0.25, (1.0 - 0.3) / 2.0):
        got = lib.selftest_limiter(a, b, kc)
        with np.errstate(divide="ignore", invalid="ignore"):
            want = kc * _superbee_reference(a / b)
        bad = np.flatnonzero(got != want)
        print(f"\n{a.size} operand pairs, kc={kc}: differing from the reference's limiter: {bad.size}")
        assert bad.size == 0, [(a[i], b[i], got[i], want[i]) for i in bad[:8]]
