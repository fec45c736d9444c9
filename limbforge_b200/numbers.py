"""numpy views of the limbforge element layout and seeded synthetic inputs.

An element ``Number<N>`` (N = bits/32) is ``N+3`` little-endian 32-bit words:
``limb[0..N-1]`` (little endian, top bit of ``limb[N-1]`` set for every nonzero value),
``exponent`` (int32), ``sign`` (int32: -1, 0, +1) and ``status`` (uint32 mask:
division_by_zero=1, exponent_overflow=2, invalid=4).  The value is
``sign * int(limbs) * 2**(exponent - (32N-1))``; zero is canonical (all words 0 apart from
a status).  ``Complex<N>`` is ``{re, im}``.  Arrays here are ``uint32`` of shape
``[count, N+3]`` (real) or ``[count, 2, N+3]`` (complex), byte-identical to the reference's
``Float<bits>`` / ``Complex<N>`` arrays (include/limbforge/core.hpp:23-34).
"""
from __future__ import annotations

import numpy as np

OK, DIVISION_BY_ZERO, EXPONENT_OVERFLOW, INVALID = 0, 1, 2, 4


def check_bits(bits: int) -> int:
    if bits < 64 or bits > 1024 or bits % 32:
        raise ValueError("bits must be a multiple of 32 in [64,1024]")
    return bits // 32


def element_words(bits: int) -> int:
    return check_bits(bits) + 3


def element_bytes(bits: int, complex_: bool = False) -> int:
    return 4 * element_words(bits) * (2 if complex_ else 1)


def zeros(count: int, bits: int, complex_: bool = False) -> np.ndarray:
    shape = (count, 2, element_words(bits)) if complex_ else (count, element_words(bits))
    return np.zeros(shape, dtype=np.uint32)


def set_fields(x: np.ndarray, exponent, sign, status=0) -> np.ndarray:
    n = x.shape[-1] - 3
    x[..., n] = np.asarray(exponent, dtype=np.int64).astype(np.int32).view(np.uint32)
    x[..., n + 1] = np.asarray(sign, dtype=np.int64).astype(np.int32).view(np.uint32)
    x[..., n + 2] = np.asarray(status, dtype=np.uint32)
    return x


def exponent(x: np.ndarray) -> np.ndarray:
    return x[..., x.shape[-1] - 3].view(np.int32)


def sign(x: np.ndarray) -> np.ndarray:
    return x[..., x.shape[-1] - 2].view(np.int32)


def status(x: np.ndarray) -> np.ndarray:
    return x[..., x.shape[-1] - 1]


def power(bits: int, e: int, sgn: int = 1, count: int = 1) -> np.ndarray:
    """sgn * 2**e"""
    n = check_bits(bits)
    x = zeros(count, bits)
    x[:, n - 1] = 0x80000000
    return set_fields(x, e, sgn)


def negate(x: np.ndarray) -> np.ndarray:
    y = x.copy()
    n = y.shape[-1] - 3
    y[..., n + 1] = (-sign(x).astype(np.int64)).astype(np.int32).view(np.uint32)
    return y


def random_numbers(rng: np.random.Generator, count: int, bits: int, span: int = 1000,
                   zero_frac: float = 0.0, sparse_frac: float = 0.0, span_lo: int | None = None) -> np.ndarray:
    """Random limbs with the top bit set, sign +-1, exponent uniform in [-span, span]
    (or [span_lo, span]); ``zero_frac`` exact zeros and ``sparse_frac`` significands with at
    most 4 set bits (the top bit and up to 3 random ones), which force exact results and ties."""
    n = check_bits(bits)
    x = np.zeros((count, n + 3), dtype=np.uint32)
    x[:, :n] = rng.integers(0, 2**32, size=(count, n), dtype=np.uint64).astype(np.uint32)
    x[:, n - 1] |= np.uint32(0x80000000)
    lo = -span if span_lo is None else span_lo
    e = rng.integers(lo, span + 1, size=count)
    s = np.where(rng.integers(0, 2, size=count) == 1, 1, -1)
    set_fields(x, e, s)
    if sparse_frac > 0:
        idx = np.nonzero(rng.random(count) < sparse_frac)[0]
        for i in idx:
            x[i, :n] = 0
            x[i, n - 1] = 0x80000000
            for _ in range(int(rng.integers(0, 4))):
                b = int(rng.integers(0, 32 * n))
                x[i, b // 32] |= np.uint32(1 << (b % 32))
    if zero_frac > 0:
        z = rng.random(count) < zero_frac
        x[z] = 0
    return x


def random_complex(rng, count, bits, span=1000, **kw) -> np.ndarray:
    re = random_numbers(rng, count, bits, span, **kw)
    im = random_numbers(rng, count, bits, span, **kw)
    return np.ascontiguousarray(np.stack([re, im], axis=1))


def to_fraction(x: np.ndarray):
    """Exact value of one real element as a Python Fraction (status elements raise)."""
    from fractions import Fraction
    n = x.shape[-1] - 3
    if int(x[n + 2]):
        raise ValueError("element carries a status")
    s = int(np.int32(x[n + 1].view(np.int32)))
    if s == 0:
        return Fraction(0)
    m = 0
    for i in range(n - 1, -1, -1):
        m = (m << 32) | int(x[i])
    e = int(x[n].view(np.int32)) - (32 * n - 1)
    return Fraction(s * m) * (Fraction(2) ** e)
