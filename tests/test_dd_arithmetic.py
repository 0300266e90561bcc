"""The double-double arithmetic of the exact-Gram mode's solves
(excalibur_b200/csrc/ddsolve.cu), restated step by step in Python floats
(IEEE double, every operation rounded on its own; the fused multiply-add
emulated exactly through rationals) and checked against exact rational
results: the error-free sums and products are exact, a double-double sum,
product with a double and quotient by a double are accurate to a few units
of 2^-104, and the compensated dot product accumulates with an error of
order (n u)^2 of the sum of |terms|."""
from fractions import Fraction as Q

import numpy as np
import pytest


def fma(a, b, c):
    return float(Q(a) * Q(b) + Q(c))


def two_sum(a, b):
    s = a + b
    bb = s - a
    return s, (a - (s - bb)) + (b - bb)


def quick_two_sum(a, b):
    s = a + b
    return s, b - (s - a)


def dd_add(x, y):
    sh, sl = two_sum(x[0], y[0])
    th, tl = two_sum(x[1], y[1])
    sl += th
    sh, sl = quick_two_sum(sh, sl)
    sl += tl
    return quick_two_sum(sh, sl)


def dd_mul_d(x, a):
    p = x[0] * a
    e = fma(x[0], a, -p) + x[1] * a
    return quick_two_sum(p, e)


def dd_div_d(x, a, ia):
    q1 = x[0] * ia
    p = q1 * a
    pe = fma(q1, a, -p)
    r = dd_add(x, (-p, -pe))
    q2 = r[0] * ia
    return quick_two_sum(q1, q2)


class Dot2:
    def __init__(self):
        self.s, self.c = 0.0, 0.0

    def add(self, a, x):
        p = a * x[0]
        pe = fma(a, x[0], -p)
        t = self.s + p
        bb = t - self.s
        self.c += ((self.s - (t - bb)) + (p - bb)) + pe + a * x[1]
        self.s = t

    def value(self):
        return quick_two_sum(self.s, self.c)


def exact(x):
    return Q(x[0]) + Q(x[1])


def rand_dd(rng, scale=1.0):
    hi = float(rng.standard_normal() * scale)
    lo = float(rng.standard_normal()) * abs(hi) * 2.0 ** -60
    return quick_two_sum(hi, lo)


U = Q(1, 2 ** 53)


def test_error_free_sum_and_product():
    rng = np.random.default_rng(1)
    for _ in range(2000):
        a, b = float(rng.standard_normal() * 10.0 ** int(rng.integers(-8, 8))), float(rng.standard_normal())
        s, e = two_sum(a, b)
        assert Q(s) + Q(e) == Q(a) + Q(b)
        p = a * b
        assert Q(p) + Q(fma(a, b, -p)) == Q(a) * Q(b)


def test_dd_add_mul_div_accuracy():
    rng = np.random.default_rng(2)
    for _ in range(2000):
        x, y = rand_dd(rng), rand_dd(rng)
        a = float(rng.standard_normal())
        if abs(a) < 1e-3:
            continue
        s = dd_add(x, y)
        bound = 4 * U * U * (abs(exact(x)) + abs(exact(y)))
        assert abs(exact(s) - (exact(x) + exact(y))) <= bound
        m = dd_mul_d(x, a)
        assert abs(exact(m) - exact(x) * Q(a)) <= 4 * U * U * abs(exact(x) * Q(a))
        q = dd_div_d(x, a, 1.0 / a)
        assert abs(exact(q) - exact(x) / Q(a)) <= 8 * U * U * abs(exact(x) / Q(a))


@pytest.mark.parametrize("n", [32, 500])
def test_compensated_dot_product(n):
    rng = np.random.default_rng(n)
    a = [float(v) for v in rng.standard_normal(n)]
    x = [rand_dd(rng) for _ in range(n)]
    d = Dot2()
    for ai, xi in zip(a, x):
        d.add(ai, xi)
    got = exact(d.value())
    want = sum(Q(ai) * exact(xi) for ai, xi in zip(a, x))
    mag = sum(abs(Q(ai) * exact(xi)) for ai, xi in zip(a, x))
    # Dot2 with the products' low parts: error ~ (n u)^2 of sum |terms| plus
    # the x.lo products' rounding (u^2 of sum |terms|)
    assert abs(got - want) <= (Q(n) ** 2 * 4 + 4 * n) * U * U * mag
