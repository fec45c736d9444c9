"""Operands of complex fused multiply-add (cfma: each component one rounding of a*b + c*d + e,
core.hpp:334-351 contract) chosen to reach every branch of a three-term exact sum: terms far apart,
products that cancel exactly or to a few bits with the addend near what is left, an addend whose
bits straddle a window's low end, two tiny terms of opposite signs below a large one, exact ties
broken by a tiny third term, and exponents near the range limits.  Generated from numpy seeds."""
import numpy as np

from limbforge_b200 import numbers as nb

KINDS = 8


def _exp(x, e):
    n = x.shape[-1] - 3
    x[..., n] = np.asarray(e, dtype=np.int64).astype(np.int32).view(np.uint32)


def dot2_cases(rng, bits, count):
    """(a, b, c) complex arrays [count, 2, N+3]; case i is of kind i % KINDS."""
    n = bits // 32
    a = nb.random_complex(rng, count, bits, 40)
    b = nb.random_complex(rng, count, bits, 40)
    c = nb.random_complex(rng, count, bits, 40)
    re, im = 0, 1
    for i in range(count):
        kind = i % KINDS
        ea = int(nb.exponent(a[i, re])) + int(nb.exponent(b[i, re]))
        if kind == 1:                                    # re: a.re b.re - a.im b.im = 0 exactly; e anywhere
            a[i, im] = a[i, re]
            b[i, im] = b[i, re]
            _exp(c[i, re], ea + int(rng.integers(-4000, 200)))
        elif kind == 2:                                  # im: a.re b.im + a.im b.re cancels to a few bits
            a[i, im] = a[i, re]
            b[i, im] = nb.negate(b[i, re][None])[0]
            b[i, im, 0] ^= np.uint32(int(rng.integers(1, 64)))
            gone = ea - 32 * n
            _exp(c[i, im], gone + int(rng.integers(-70, 70)))
            _exp(c[i, re], ea - 64 * n + int(rng.integers(-30, 30)))
        elif kind == 3:                                  # the addend straddles a 3N+4-word window's low end
            _exp(a[i, im], int(nb.exponent(a[i, im])) - int(rng.integers(0, 40)))
            _exp(c[i, re], ea - 96 * n - 125 + int(rng.integers(-64, 65)))
            _exp(c[i, im], ea - 64 * n - int(rng.integers(0, 200)))
        elif kind == 4:                                  # two tiny terms of opposite signs below a large one
            _exp(a[i, im], int(nb.exponent(a[i, im])) - 100 * n - 300)
            _exp(c[i, re], ea - 100 * n - 300 + int(rng.integers(-3, 4)))
            s = int(nb.sign(a[i, im])) * int(nb.sign(b[i, im]))     # -a.im b.im has sign -s: give e the sign s
            c[i, re, n + 1] = np.int32(s).view(np.uint32)
        elif kind == 5:                                  # an exact tie broken (or not) by a tiny product
            a[i, re] = nb.power(bits, int(rng.integers(-20, 20)))[0]
            b[i, re] = nb.power(bits, int(rng.integers(-20, 20)))[0]
            b[i, re, 0] |= np.uint32(1)                  # a.re b.re = 2^x (1 + 2^(1-32N)): exact, odd last place
            top = int(nb.exponent(a[i, re])) + int(nb.exponent(b[i, re]))
            c[i, re] = nb.power(bits, top - 32 * n, int(rng.choice([-1, 1])))[0]     # half a unit: a tie
            if rng.integers(0, 2):
                a[i, im] = 0
            else:
                _exp(a[i, im], top - 40 * n - 500)
        elif kind == 6:                                  # exponents near the range limit
            big = 500000000 - int(rng.integers(0, 3))
            _exp(a[i, re], big)
            _exp(b[i, re], big)
            _exp(a[i, im], -big)
            _exp(c[i, re], int(rng.integers(-50, 50)))
        elif kind == 7:                                  # one product zero, the other two terms cancelling
            a[i, im] = 0
            c[i, re] = nb.negate(a[i, re][None])[0]
            b[i, re] = nb.power(bits, 0)[0]
            c[i, re, 0] ^= np.uint32(int(rng.integers(0, 2)))
    return a, b, c
