"""The exact-sum arithmetic of the device kernels, restated on the host.

Every sum of the library (kept mass, total mass, sum of |a|^4, RDM moments,
norm, PR) is the sum of floor(|v| * 2^96) * sign(v) over its terms
(``fx_from`` in ``csrc/common.cuh`` and ``oracle/bass_oracle.c``).  The hot
sums on the device form that integer as h * 2^48 + l with h and l exact
integer-valued doubles (``fx_split96``) and add up to eight of them in
floating point before joining (``fx_join96`` / ``fx_join96s``).  Python
floats are IEEE doubles with the same round-to-nearest operations, so this
checks the arithmetic itself: the split is exact and eight-term sums of the
parts stay exact.
"""
import math
import random
from fractions import Fraction

import pytest

TWO96, TWO48, TWOM48 = 2.0 ** 96, 2.0 ** 48, 2.0 ** -48


def fx_exact(v: float) -> int:
    """floor(|v| * 2^96), negated for v < 0 (the definition)."""
    m = math.floor(Fraction(abs(v)) * 2 ** 96)
    return -m if v < 0 else m


def split96(v: float):
    """fx_split96 of |v| with the device's operations, signs applied after."""
    a = abs(v)
    x = a * TWO96
    h = math.trunc(x * TWOM48) * 1.0
    l = math.trunc(x - h * TWO48) * 1.0
    if v < 0:
        h, l = -h, -l
    return h, l


def sample_values(rng, n):
    out = []
    for i in range(n):
        e = rng.randint(0, 140)
        v = rng.random() * 2.0 ** -e
        if i % 7 == 0:
            v = 2.0 - 2.0 ** -52 * rng.randint(1, 50)      # just below 2
        if i % 11 == 0:
            v = 2.0 ** -rng.randint(0, 100)                 # powers of two
        if i % 13 == 0:
            v = 2.0 ** -96 * rng.random()                   # below the resolution
        if i % 3 == 0:
            v = -v
        out.append(v)
    return out + [0.0, -0.0, 5e-324, 2.0 ** -96, 1.0, 1.9999999999999998]


def test_split_is_exact():
    rng = random.Random(1)
    for v in sample_values(rng, 20000):
        h, l = split96(v)
        assert h == math.trunc(h) and l == math.trunc(l)
        assert abs(h) < 2.0 ** 50 and abs(l) < 2.0 ** 48
        assert int(h) * 2 ** 48 + int(l) == fx_exact(v), v


@pytest.mark.parametrize("signed", [False, True])
def test_eight_term_sums_stay_exact(signed):
    rng = random.Random(2 + signed)
    vals = sample_values(rng, 8000)
    if not signed:
        vals = [abs(v) for v in vals]
    for k in range(0, len(vals) - 8, 8):
        chunk = vals[k:k + 8]
        dh = dl = 0.0
        for v in chunk:
            h, l = split96(v)
            dh += h
            dl += l
        # the doubles hold the exact integer sums (no rounding happened)
        assert dh == sum(int(split96(v)[0]) for v in chunk)
        assert dl == sum(int(split96(v)[1]) for v in chunk)
        assert int(dh) * 2 ** 48 + int(dl) == sum(fx_exact(v) for v in chunk)
