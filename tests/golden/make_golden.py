"""Generates the golden vectors under tests/golden/ (run from the repository root with the
reference checkout present: ``python tests/golden/make_golden.py``).

Inputs follow the fixture classes of the reference's own tests, regenerated here with numpy
seeds (the reference stores no vectors; it recomputes everything with MPFR):

* real ops (tests/test_arithmetic.cpp:16-75): random operands, forced cancellation and ulp
  alignment, halfway ties, deep exact cancellation, exponent-limit overflow/underflow, all-ones
  significands, exact products just below a binade that rounding rescues from emin-1, and
  square-root inputs next to root rounding boundaries of both exponent parities;
* fused ops (tests/test_fused.cpp:10-27): the 23 fma/fms classes and the 11 complex-fma classes;
* exact dots (tests/test_linalg.cpp:22-68): random spans, exact and near cancellation, ties
  created by far terms and by the addend, last-bit cancellation and exponent limits.

Expected outputs come from the reference's CPU arithmetic compiled from its sources
(oracle/_ref/libref.so: core.hpp and linalg.hpp::exact_dot_add); generation fails unless MPFR
(oracle/libmpfr_oracle.so) agrees bit for bit on every canonical case.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from limbforge_b200 import numbers as nb  # noqa: E402
from oracle.oracle import Mpfr, Reference, build  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
WIDTHS = [64, 96, 128, 224, 256, 384, 512, 1024]


def from_int(bits, m: int, exponent: int, sign: int) -> np.ndarray:
    """element with significand integer m (top bit at 32N-1)"""
    n = bits // 32
    x = np.zeros(n + 3, dtype=np.uint32)
    for i in range(n):
        x[i] = (m >> (32 * i)) & 0xffffffff
    nb.set_fields(x, exponent, sign)
    return x


def to_int(x: np.ndarray) -> int:
    n = x.shape[-1] - 3
    m = 0
    for i in range(n - 1, -1, -1):
        m = (m << 32) | int(x[i])
    return m


def one(bits, e=0, sign=1):
    return from_int(bits, 1 << (bits - 1), e, sign)


def real_cases(bits: int, rng: np.random.Generator, count: int = 256):
    n = bits // 32
    a = nb.random_numbers(rng, count, bits, 1000)
    b = nb.random_numbers(rng, count, bits, 1000)
    for i in range(count):
        if i % 3 == 0:
            b[i, n] = np.int32(int(nb.exponent(a[i])) - int(rng.integers(0, bits + 80))).view(np.uint32)
        if i % 11 == 0:
            b[i] = nb.negate(a[i][None])[0]
            b[i, 0] ^= np.uint32(rng.integers(0, 256))
        if i % 17 == 0:
            a[i] = 0
        if i % 23 == 0:
            b[i] = 0
        if i % 101 == 0 and i:
            a[i, n + 2] = nb.INVALID
    a[1], b[1] = one(bits), one(bits, -bits)                          # 1 + half ulp: tie, stays even
    a[2], b[2] = one(bits), one(bits, -bits)
    a[2, 0] |= 1                                                      # odd: rounds up
    a[3], b[3] = one(bits), one(bits, -bits, -1)                      # binade boundary
    a[4], b[4] = one(bits), one(bits, 0, -1)
    a[4, 0] = 1                                                       # deep exact cancellation
    a[5], b[5] = one(bits, 1000000000), one(bits, 1)                  # overflow
    a[6], b[6] = one(bits, -1000000000), one(bits, -1)                # underflow
    a[7] = from_int(bits, (1 << bits) - 1, 0, 1)
    b[7] = from_int(bits, (1 << bits) - 1, 0, 1)
    # exact products just below a binade boundary: rounding can rescue emin-1
    target, half = 1 << (2 * bits - 1), 1 << (bits - 2)
    for f in range(8, 40):
        while True:
            za = int(rng.integers(0, 2**63)) | (1 << 63)
            za = (za << (bits - 64)) | int(rng.integers(0, 2**62)) if bits > 64 else za
            za |= 1 << (bits - 1)
            za &= (1 << bits) - 1
            zb, rem = divmod(target, za)
            if rem and rem < half and zb.bit_length() == bits:
                break
        sgn = -1 if f % 2 else 1
        ea, eb = (-1000000000, -1) if f % 3 else (1000000000, 0)
        a[f] = from_int(bits, za, ea, sgn)
        b[f] = from_int(bits, zb, eb, sgn)
    roots = a.copy()
    roots[0] = 0
    roots[1], roots[2], roots[3] = one(bits), one(bits, 1), one(bits, 2)
    for f in range(40, 104):
        q = int(rng.integers(0, 2**63)) | (1 << 63)
        q = (q << (bits - 64)) | int(rng.integers(0, 2**62)) if bits > 64 else q
        q |= 1 << (bits - 1)
        q &= (1 << bits) - 1
        zb = q * q + q                                                 # floor((q+1/2)^2)
        parity = int(zb.bit_length() == 2 * bits)
        zb >>= bits - 1 + parity
        if f % 2:
            zb += 1
        if zb.bit_length() > bits:
            zb -= 1
        roots[f] = from_int(bits, zb, parity - (0 if f % 3 else 2), 1)
    roots[:, n + 1] = np.abs(nb.sign(roots)).astype(np.int32).view(np.uint32)
    return a, b, roots


def half_ulp(bits, x, sign):
    return one(bits, int(nb.exponent(x)) - bits, sign)


def fused_cases(bits: int, rng: np.random.Generator, count: int = 230, ref=None):
    n = bits // 32
    a = nb.random_numbers(rng, count, bits, 40)
    b = nb.random_numbers(rng, count, bits, 40)
    c = nb.random_numbers(rng, count, bits, 80)
    prod = ref.elementwise(bits, 2, a, b)
    for i in range(count):
        k = i % 23
        if k == 0:
            c[i] = nb.negate(prod[i][None])[0]
        elif k == 1:
            c[i] = nb.negate(prod[i][None])[0]
            c[i, 0] ^= np.uint32(rng.integers(0, 16))
        elif k == 2:
            c[i, n] = np.int32(int(nb.exponent(a[i])) + int(nb.exponent(b[i])) - int(rng.integers(0, 3 * bits + 80))).view(np.uint32)
        elif k == 3:
            c[i, n] = np.int32(int(nb.exponent(a[i])) + int(nb.exponent(b[i])) + int(rng.integers(0, 2 * bits + 80))).view(np.uint32)
        elif k in (4, 5):
            a[i] = one(bits)
            c[i] = half_ulp(bits, b[i], 1 if rng.integers(0, 2) else -1)
            if k == 5:
                c[i, 0] |= 1
        elif k == 6:
            a[i] = 0
        elif k == 7:
            c[i] = 0
        elif k == 8:
            b[i] = 0
            c[i] = 0
        elif k == 9:
            c[i, n + 2] = nb.INVALID
        elif k in (10, 11):
            a[i, n] = np.int32(600000000).view(np.uint32)
            b[i, n] = np.int32(600000000).view(np.uint32)
            if k == 10:
                c[i] = nb.negate(ref.elementwise(bits, 2, a[i:i + 1], b[i:i + 1]))[0]
            else:
                c[i, n] = np.int32(999999990).view(np.uint32)
        elif k == 12:
            a[i, n] = np.int32(-600000000).view(np.uint32)
            b[i, n] = np.int32(-500000000).view(np.uint32)
            c[i, n] = np.int32(-999999999).view(np.uint32)
        elif k == 13:
            a[i, n] = 0
            b[i, n] = 0
            c[i] = nb.negate(a[i][None])[0]
            c[i, n] = 0
    return a, b, c


def complex_fused_cases(bits: int, rng: np.random.Generator, count: int = 132, ref=None):
    n = bits // 32
    A = nb.random_complex(rng, count, bits, 30)
    B = nb.random_complex(rng, count, bits, 30)
    Cc = nb.random_complex(rng, count, bits, 60)
    for i in range(count):
        k = i % 11
        if k in (0, 1):
            B[i, 0], B[i, 1] = A[i, 1].copy(), A[i, 0].copy()
            if k == 1:
                B[i, 0, 0] ^= 1
        elif k == 2:
            A[i, 0] = one(bits)
            Cc[i, 0] = nb.negate(B[i, 0][None])[0]
            A[i, 1, n] = np.int32(-3 * bits).view(np.uint32)
            B[i, 1, n] = np.int32(-3 * bits).view(np.uint32)
        elif k == 3:
            p = ref.elementwise(bits, 5, A[i:i + 1], B[i:i + 1])
            Cc[i, 0] = nb.negate(p[:, 0])[0]
            Cc[i, 1] = nb.negate(p[:, 1])[0]
        elif k == 4:
            A[i, 1, n] = np.int32(int(nb.exponent(A[i, 1])) - int(rng.integers(0, 4 * bits))).view(np.uint32)
        elif k == 5:
            Cc[i, 0, n] = np.int32(int(nb.exponent(Cc[i, 0])) - int(rng.integers(0, 4 * bits))).view(np.uint32)
            Cc[i, 1, n] = np.int32(int(nb.exponent(Cc[i, 1])) + int(rng.integers(0, 4 * bits))).view(np.uint32)
        elif k == 6:
            A[i, 1] = 0
        elif k == 7:
            Cc[i] = 0
        elif k == 8:
            A[i, 0] = one(bits)
            A[i, 1] = 0
            Cc[i, 0] = half_ulp(bits, B[i, 0], -1)
    return A, B, Cc


def dot_cases(bits: int, rng: np.random.Generator):
    """list of (a [K,E], b [K,E], c [E] or None, subtract)"""
    n = bits // 32
    cases = []
    pw = lambda e, s=1: one(bits, e, s)
    for it in range(24):
        K = 1 + int(rng.integers(0, 40))
        span = [5, 300, 3000, 900000000][it % 4]
        a = nb.random_numbers(rng, K, bits, span)
        b = nb.random_numbers(rng, K, bits, span // 2 + 1)
        a[rng.random(K) < 1 / 9] = 0
        if it % 5 == 1:
            a[K - 1], b[K - 1] = nb.negate(a[0][None])[0], b[0]
        if it % 5 == 2 and K > 2:
            a[1], b[1] = nb.negate(a[0][None])[0], b[0]
            a[2, n] = np.int32(int(nb.exponent(a[0])) - 4 * bits).view(np.uint32)
        if it % 7 == 3:
            a[int(rng.integers(0, K)), n + 2] = nb.INVALID
        for sub in (False, True):
            cases.append((a, b, None, sub))
            cases.append((a, b, nb.random_numbers(rng, 1, bits, 40)[0], sub))
    odd = one(bits)
    odd[0] |= 1
    for s in (1, -1):
        for p in (1, bits // 2, bits - 1):
            for extra in (0, 1, -1):
                a = np.stack([one(bits), pw(-p, s), pw(700), pw(700, -1), odd])
                b = np.stack([pw(0, s), pw(-(bits - p) - extra), pw(-3), pw(-3), np.zeros(n + 3, np.uint32)])
                cases.append((a, b, None, False))
                a2 = a.copy(); a2[0] = odd
                cases.append((a2, b, None, False))
                a3 = a2.copy(); a3[2] = pw(9000); a3[3] = pw(9000, -1)
                cases.append((a3, b, None, False))
                b4 = b.copy(); b4[4] = pw(-(2 * bits + 500), -s)
                cases.append((a3, b4, None, False))
    two = one(bits)
    two[0] |= 2
    for s in (1, -1):
        for d in (1, 20, bits - 2, bits - 1, bits, bits + 1, bits + 6, bits + 40, 3 * bits):
            a = np.stack([odd, one(bits), pw(2 - 2 * bits - d)])
            b = np.stack([odd, nb.negate(two[None])[0], pw(0, s)])
            cases.append((a, b, None, False))
            a2 = np.concatenate([a, pw(2 - 2 * bits - d - bits - 9)[None]])
            b2 = np.concatenate([b, pw(0, -s)[None]])
            cases.append((a2, b2, None, False))
    for s in (1, -1):
        for c in (one(bits), odd):
            c = c if s > 0 else nb.negate(c[None])[0]
            cases.append((pw(-bits)[None], pw(0, -s)[None], c, True))
            cases.append((np.stack([pw(-bits), pw(-3 * bits)]), np.stack([pw(0, -s), pw(0, s)]), c, True))
            cases.append((np.stack([pw(-bits), pw(-3 * bits)]), np.stack([pw(0, -s), pw(0, -s)]), c, True))
            cases.append((np.stack([pw(500), pw(500), pw(-bits)]), np.stack([pw(2), pw(2, -1), pw(0, -s)]), c, True))
    a = np.stack([pw(600000000), pw(-600000000)])
    b = np.stack([pw(500000000), pw(-500000000)])
    cases.append((a, b, None, False))
    a = np.stack([pw(-600000000), pw(-600000000)])
    b = np.stack([pw(-400000000), pw(-500000000)])
    cases.append((a, b, None, False))
    a2 = a.copy(); a2[0, 0] = 0xffffffff
    cases.append((a2, b, None, False))
    cases.append((np.zeros((0, n + 3), np.uint32), np.zeros((0, n + 3), np.uint32), None, False))
    return cases


def main():
    build()
    ref, mp = Reference(), Mpfr()
    rng = np.random.default_rng(20261203)
    out = {}
    for bits in WIDTHS:
        a, b, roots = real_cases(bits, rng)
        for op in (0, 1, 2, 3, 7, 8):
            x = roots if op == 8 else a
            want = ref.elementwise(bits, op, x, b)
            canon = (nb.status(x) == 0) & ((nb.sign(x) != 0) | (x[:, :-1].max(axis=1) == 0))
            if op not in (7, 8):
                canon &= (nb.status(b) == 0)
            m = mp.real(bits, op, x, b)
            bad = np.nonzero(canon & (m != want).any(axis=1))[0]
            assert not len(bad), f"MPFR disagrees with the reference: bits={bits} op={op} cases={bad[:5]}"
            out[f"real_{bits}_{op}_out"] = want
        out[f"real_{bits}_a"], out[f"real_{bits}_b"], out[f"real_{bits}_roots"] = a, b, roots
        fa, fb, fc = fused_cases(bits, rng, ref=ref)
        for op in (9, 10):
            want = ref.elementwise(bits, op, fa, fb, fc)
            m = mp.fused(bits, op == 10, fa, fb, fc)
            assert (m == want).all(), f"MPFR fma disagrees: bits={bits}"
            out[f"fused_{bits}_{op}_out"] = want
        out[f"fused_{bits}_a"], out[f"fused_{bits}_b"], out[f"fused_{bits}_c"] = fa, fb, fc
        ca, cb, cc = complex_fused_cases(bits, rng, ref=ref)
        for op in (4, 5, 6, 11, 12):
            want = ref.elementwise(bits, op, ca, cb, cc)
            if op in (4, 5, 6):
                assert (mp.complex(bits, op, ca, cb) == want).all(), f"MPFR complex disagrees: bits={bits} op={op}"
            out[f"cx_{bits}_{op}_out"] = want
        out[f"cx_{bits}_a"], out[f"cx_{bits}_b"], out[f"cx_{bits}_c"] = ca, cb, cc
        E = bits // 32 + 3
        for q, (da, db, dc, sub) in enumerate(dot_cases(bits, rng)):
            K = da.shape[0]
            A = np.ascontiguousarray(da, dtype=np.uint32)
            B = np.ascontiguousarray(db, dtype=np.uint32)
            cc_ = None if dc is None else np.ascontiguousarray(dc, dtype=np.uint32)
            want = ref.exact_dot_add(bits, cc_, sub, A, 1, B, 1, K)
            m = mp.dot(bits, cc_, sub, A, 1, B, 1, K)
            # MPFR returns RN(c) for a c with no nonzero product; the reference returns c itself
            if not ((nb.status(A) != 0).any() or (nb.status(B) != 0).any()):
                assert (m == want).all(), f"MPFR dot disagrees: bits={bits} case={q}"
            out[f"dot_{bits}_{q}_a"], out[f"dot_{bits}_{q}_b"] = A, B
            out[f"dot_{bits}_{q}_c"] = np.zeros(E, np.uint32) if cc_ is None else cc_
            out[f"dot_{bits}_{q}_meta"] = np.array([int(cc_ is not None), int(sub)], dtype=np.uint32)
            out[f"dot_{bits}_{q}_out"] = want
    np.savez_compressed(os.path.join(OUT, "arith_golden.npz"), **out)
    print(f"wrote {len(out)} arrays to {OUT}/arith_golden.npz")


if __name__ == "__main__":
    main()
