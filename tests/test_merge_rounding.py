"""CPU check of the coalescence arithmetic used by the merge kernel
(particle-simulator_b200/csrc/merge.cu): r^3 and v^RN(1/3) computed from
error-free products, a Newton correction of the cube root and a first-order
correction for the exponent RN(1/3) = 1/3 - 2^-54/3 are correctly rounded.

The kernel's formulas are evaluated here with exact rational arithmetic for
each fused multiply-add and compared with 60-digit decimal arithmetic.  The
same comparison shows that libm's pow (which numpy, and therefore the
reference, calls) is not correctly rounded in a small fraction of cases."""

from __future__ import annotations

import math
from decimal import Decimal, getcontext
from fractions import Fraction as Fr

import numpy as np

getcontext().prec = 60
E = 1.0 / 3.0


def fma(x, y, z):
    return float(Fr(x) * Fr(y) + Fr(z))


def cube_rn(x):
    p = x * x
    e = fma(x, x, -p)
    return fma(x, p, x * e)


def pow_third_rn(v):
    c0 = float(np.cbrt(v))
    ph = c0 * c0
    pl = fma(c0, c0, -ph)
    qh = c0 * ph
    ql = fma(c0, ph, -qh)
    res = ((v - qh) - ql) - c0 * pl
    corr = res / (3.0 * ph)
    kappa = -(2.0**-54 / 3.0) * math.log(v)
    return c0 + (corr + c0 * kappa)


def exact_pow(v, e):
    fe = Fr(e)
    val = (Decimal(fe.numerator) / Decimal(fe.denominator) * Decimal(v).ln()).exp()
    return float(Fr(val))


def test_exponent_offset():
    assert Fr(1, 3) - Fr(E) == Fr(1, 3 * 2**54)


def test_cube_and_cube_root_correctly_rounded():
    rng = np.random.default_rng(5)
    r = np.exp(rng.uniform(np.log(1e-7), np.log(1e-3), 3000))
    libm_off = 0
    for a, b in zip(r[0::2], r[1::2]):
        a, b = float(a), float(b)
        assert cube_rn(a) == float(Fr(a) ** 3)
        v = cube_rn(a) + cube_rn(b)
        ex = exact_pow(v, E)
        assert pow_third_rn(v) == ex
        libm_off += (v**E) != ex
    assert libm_off < 20  # libm pow: rarely, but not never, off by one ulp
