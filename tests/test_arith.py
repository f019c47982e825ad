"""Arithmetic identities the kernels rely on, checked on the CPU.

The image preparation divides each gradient numerator by 12 as the quotient
by the rounded reciprocal plus one FMA correction (prep.cu, div12) instead of
an IEEE division. For this to leave the planes bit-identical to the CPU
restatement (which divides), the two must agree for every numerator an 8-bit
image can produce: -I[x+2] + 8 I[x+1] - 8 I[x-1] + I[x-2] lies within
|x| <= 9 * 255 = 2295. Checked here with exact rational arithmetic and correct
float32 rounding.
"""
from fractions import Fraction

import numpy as np


def _rn32(fr: Fraction) -> np.float32:
    """The float32 nearest to an exact rational (ties to even)."""
    c = np.float32(float(fr))
    best = None
    for cand in (np.nextafter(c, np.float32(-np.inf)), c, np.nextafter(c, np.float32(np.inf))):
        d = abs(Fraction(float(cand)) - fr)
        even = (int(np.frombuffer(cand.tobytes(), np.uint32)[0]) & 1) == 0
        if best is None or d < best[0] or (d == best[0] and even):
            best = (d, cand)
    return best[1]


def _fma(a, b, c) -> np.float32:
    return _rn32(Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c)))


def test_division_by_12_correction_is_exact():
    inv = np.float32(1.0) / np.float32(12.0)
    for num in range(-2295, 2296):
        x = np.float32(num)
        q = _rn32(Fraction(float(x)) * Fraction(float(inv)))
        r = _fma(-q, np.float32(12.0), x)
        q2 = _fma(r, inv, q)
        ieee = x / np.float32(12.0)
        assert q2 == ieee and np.signbit(q2) == np.signbit(ieee), num
