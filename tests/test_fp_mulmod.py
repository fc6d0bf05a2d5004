"""The double-precision modular product of via_rs_b200/csrc/ntt_fp.cuh, checked on the host,
and the scan epilogue's fold of nine accumulator groups built on it (fd_tc.cu fold9).

fp_mulmod(a, b) computes, with IEEE-754 double operations rounded to nearest:
    ph = a * b;  pl = fma(a, b, -ph);  qt = (fma(ph, qinv, R) - R);  r = fma(-qt, q, ph) + pl
with R = 1.5 * 2^52 and qinv the rounded 1/q. The claim the transforms rely on: for
integers |a| < 2^48 and 0 <= b < q (q below 2^44), r is an integer, r = a * b (mod q),
and |r| <= 0.5625 q. Python floats are IEEE doubles; an FMA is a single rounding of the
exact a * b + c, restated here with exact rationals. No GPU needed.
"""
from fractions import Fraction

import numpy as np
import pytest

R = 6755399441055744.0  # 1.5 * 2^52


def fma(a: float, b: float, c: float) -> float:
    return float(Fraction(a) * Fraction(b) + Fraction(c))  # exact, then one rounding to nearest even


def fp_mulmod(a: float, b: float, q: float, qinv: float) -> float:
    ph = a * b
    pl = fma(a, b, -ph)
    qt = fma(ph, qinv, R) - R
    return fma(-qt, q, ph) + pl


def fp_canonical(x: float, q: float, qinv: float) -> float:
    qt = fma(x, qinv, R) - R
    r = fma(-qt, q, x)
    if r < 0:
        r += q
    if r >= q:
        r -= q
    return r


# q2, the two q1 primes, q3, and a modulus near the 2^44 limit (the claim holds for any modulus).
MODULI = [17175674881, 137438822401, 274810798081, 8380417, (1 << 43) - 14 * 8192 + 1]


@pytest.mark.parametrize("q", MODULI)
def test_products_exact_and_within_bound(q):
    qd, qinv = float(q), 1.0 / float(q)
    rng = np.random.default_rng(q % 1000)
    amax = 1 << 48
    cases = [(int(x), int(y)) for x, y in zip(rng.integers(-amax + 1, amax, size=3000), rng.integers(0, q, size=3000))]
    cases += [(amax - 1 - k, q - 1 - k) for k in range(50)] + [(-(amax - 1) + k, q - 1 - k) for k in range(50)]
    cases += [(k, q - 1) for k in range(-50, 50)]
    worst = 0.0
    for a, b in cases:
        r = fp_mulmod(float(a), float(b), qd, qinv)
        assert r == int(r)
        assert (a * b - int(r)) % q == 0, (q, a, b, r)
        worst = max(worst, abs(r) / q)
    assert worst <= 0.5625, worst


@pytest.mark.parametrize("q", MODULI)
def test_canonical_reduction(q):
    qd, qinv = float(q), 1.0 / float(q)
    rng = np.random.default_rng(7)
    for x in list(rng.integers(-(1 << 50) + 1, 1 << 50, size=2000)) + [0, q, -q, q - 1, 1 - q, 8 * q, -8 * q]:
        r = fp_canonical(float(int(x)), qd, qinv)
        assert 0 <= r < q and (int(x) - int(r)) % q == 0


def fold9(v, q):
    """fd_tc.cu fold9: sum_g v_g 2^(8g) mod q from the groups 0-2, 3-5, 6-8."""
    qd, qinv = float(q), 1.0 / float(q)
    lo = v[0] + (v[1] << 8) + (v[2] << 16)
    m1 = v[3] + (v[4] << 8) + (v[5] << 16)
    m2 = v[6] + (v[7] << 8) + (v[8] << 16)
    assert max(lo, m1, m2) < 1 << 48
    r1 = fp_mulmod(float(m1), float((1 << 24) % q), qd, qinv)
    r2 = fp_mulmod(float(m2), float((1 << 48) % q), qd, qinv)
    return fp_canonical((float(lo) + r1) + r2, qd, qinv)


@pytest.mark.parametrize("q", [m for m in MODULI if m < 1 << 40] + [1_099_511_480_321])
def test_fold9_exact(q):
    """Group sums below 2^31 (the TMEM accumulators of a scan over at most 4096 rows)."""
    rng = np.random.default_rng(q % 4093)
    top = (1 << 31) - 1
    cases = [[int(x) for x in row] for row in rng.integers(0, 1 << 31, size=(3000, 9))]
    cases += [[top] * 9, [0] * 9, [1] * 9, [top if g % 2 else 0 for g in range(9)], [0] * 8 + [top]]
    for v in cases:
        want = sum(x << (8 * g) for g, x in enumerate(v)) % q
        got = fold9(v, q)
        assert got == want, (q, v, got, want)
