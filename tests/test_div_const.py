"""The constant-divisor quotient of the kernels (div_const in
opencaeporo_b200/csrc/flash_common.cuh): q = RN(x rd), r = fma(-d, q, x),
result fma(r, rd, q) with rd = RN(1/d). Its claim is bit equality with the
IEEE quotient x / d. This test replays the three steps in exact rational
arithmetic (an FMA rounds once: RN of the exact value) and checks that the
remainder is exact and that the result equals Python's correctly rounded
x / d, for the divisors the kernels use, on random magnitudes over the whole
fast-path range and on quotients next to powers of two, where one ulp is
largest relative to the quotient."""
from fractions import Fraction

import numpy as np
import pytest

D1 = 2.41421356237
D2 = -0.41421356237
DIVISORS = {"3": 3.0, "9": 9.0, "54": 54.0, "d1-d2": D1 - D2}


def _fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def _div_const(x, d, rd):
    ax = abs(x)
    if not (1e-270 < ax < 1e270):
        return x / d
    q = x * rd
    rex = Fraction(x) - Fraction(d) * Fraction(q)
    r = float(rex)
    assert Fraction(r) == rex, "remainder not exact"
    return _fma(r, rd, q)


def _samples(d, n, seed):
    rng = np.random.default_rng(seed)
    # magnitudes spread over the fast-path range, random signs and mantissas
    e = rng.uniform(-268, 268, n)
    x = np.sign(rng.uniform(-1, 1, n)) * 10.0 ** e
    # quotients at and next to powers of two: x = d 2^k (1 + j ulp)
    k = rng.integers(-800, 800, n // 4)
    j = rng.integers(-64, 65, n // 4)
    y = d * np.ldexp(1.0, k) * (1 + j * 2.0 ** -52)
    # mantissas with long runs of ones and zeros
    m = np.ldexp(np.float64(2 ** 53 - 1), -52) * np.ldexp(1.0, rng.integers(-300, 300, n // 8))
    z = np.concatenate([m, np.nextafter(m, 0), np.nextafter(m, 4 * m)])
    return np.concatenate([x, y, z, [1.0, -1.0, d, -d, 3 * d, 0.0, -0.0]])


@pytest.mark.parametrize("name", list(DIVISORS))
def test_div_const_is_the_correctly_rounded_quotient(name):
    d = DIVISORS[name]
    rd = 1.0 / d
    xs = _samples(d, 20000, sum(map(ord, name)))
    bad = []
    for x in xs:
        x = float(x)
        got = _div_const(x, d, rd)
        want = x / d
        if not (got == want and np.signbit(got) == np.signbit(want)):
            bad.append((x, got, want))
    assert not bad, bad[:5]
