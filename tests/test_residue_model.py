"""CPU: a Python-integer model of the residue/CRT engine's arithmetic (lf_residue.cuh) checked
against the oracle's exact dot products.  It pins the algorithm the kernels implement: the
modulus count rule, balanced residues split into two int8 digits, the three int8 products
65536 S11 + 256 Smid + S00, the CRT with the fixed-point rounding of the quotient, and the single
final rounding of c - X 2^scale.  The kernels themselves are checked on the GPU."""
import math

import numpy as np
import pytest

from limbforge_b200 import numbers as nb


def primes_desc(count, top=65279):
    out, q = [], top
    while len(out) < count:
        if q > 1 and all(q % d for d in range(2, int(q ** 0.5) + 1)):
            out.append(q)
        q -= 1
    return out


def aligned(x, bottom, n):
    m = 0
    for i in range(n - 1, -1, -1):
        m = (m << 32) | int(x[i])
    s = int(np.int32(x[n + 1].view(np.int32)))
    e = int(x[n].view(np.int32))
    return s * (m << (e - bottom)) if s else 0


def model_dot(bits, A, B, K, drop=0):
    """X = sum_k a_k b_k as the engine computes it, plus its scale (drop: use that many moduli fewer than the
    count rule gives, to show the rule is needed)."""
    n = bits // 32
    ea = [int(v) for v in nb.exponent(A[nb.sign(A) != 0])]
    eb = [int(v) for v in nb.exponent(B[nb.sign(B) != 0])]
    ba, bb = min(ea), min(eb)
    G = max(max(ea) - ba, max(eb) - bb)
    P = 32 * n + G
    need = 2 * P + math.ceil(math.log2(max(K, 2))) + 3
    mods, have = [], 0.0
    for m in primes_desc(200):
        if have > need:
            break
        mods.append(m)
        have += math.log2(m)
    mods = mods[:len(mods) - drop]
    X = [aligned(A[k], ba, n) for k in range(K)]
    Y = [aligned(B[k], bb, n) for k in range(K)]
    residues = []
    for m in mods:
        def digits(v):
            r = v % m
            if r > m // 2:
                r -= m
            lo = ((r & 0xff) ^ 0x80) - 0x80
            hi = (r - lo) >> 8
            assert -128 <= lo <= 127 and -128 <= hi <= 127
            return hi, lo
        s11 = s00 = smid = 0
        for k in range(K):
            h1, l1 = digits(X[k])
            h2, l2 = digits(Y[k])
            s11 += h1 * h2
            s00 += l1 * l2
            smid += h1 * l2 + l1 * h2
        for s in (s11, s00, smid):
            assert -2**31 <= s < 2**31
        residues.append((65536 * s11 + 256 * smid + s00) % m)
    M = math.prod(mods)
    S = F = 0
    for m, r in zip(mods, residues):
        q = M // m
        t = r * pow(q % m, -1, m) % m
        S += t * q
        F += t * ((1 << 48) // m)
    qround = (F + (1 << 47)) >> 48
    return S - qround * M, ba + bb - 2 * (32 * n - 1), len(mods)


@pytest.mark.parametrize("bits,K,span", [(64, 1, 3), (128, 17, 40), (256, 64, 40), (512, 9, 80), (96, 33, 0)])
def test_residue_model_is_exact(oracle, bits, K, span):
    from fractions import Fraction
    rng = np.random.default_rng(bits + K)
    n = bits // 32
    A = nb.random_numbers(rng, K, bits, span)
    B = nb.random_numbers(rng, K, bits, span)
    X, scale, L = model_dot(bits, A, B, K)
    exact = sum((nb.to_fraction(A[k]) * nb.to_fraction(B[k]) for k in range(K)), Fraction(0))
    assert Fraction(X) * Fraction(2) ** scale == exact
    # the single rounding of c - X 2^scale equals the oracle's exact_dot_add
    c = nb.random_numbers(rng, 1, bits, span)[0]
    want = oracle.exact_dot_add(bits, c, 1, A, 1, B, 1, K)
    val = nb.to_fraction(c) - Fraction(X) * Fraction(2) ** scale
    if val == 0:
        assert int(nb.sign(want)) == 0
    else:
        assert nb.to_fraction(want) == round_fraction(val, bits)


def round_fraction(v, bits):
    """RN to `bits` significant bits, ties to even (reference value for the test)."""
    from fractions import Fraction
    s = -1 if v < 0 else 1
    v = abs(v)
    e = v.numerator.bit_length() - v.denominator.bit_length()
    while Fraction(2) ** e > v:
        e -= 1
    while Fraction(2) ** (e + 1) <= v:
        e += 1
    q = v / Fraction(2) ** (e - bits + 1)
    fl = q.numerator // q.denominator
    rem = q - fl
    if rem > Fraction(1, 2) or (rem == Fraction(1, 2) and fl % 2):
        fl += 1
    return s * Fraction(fl) * Fraction(2) ** (e - bits + 1)


def test_digit_split_bounds():
    """Balanced residues modulo primes <= 65279 always split into two int8 digits; 65281 would not."""
    for m in (65279, 65267, 40009):
        for r in (-(m - 1) // 2, (m - 1) // 2, -32639, 127, -128):
            if abs(r) > (m - 1) // 2:
                continue
            lo = ((r & 0xff) ^ 0x80) - 0x80
            hi = (r - lo) >> 8
            assert -128 <= hi <= 127
    r = (65521 - 1) // 2
    lo = ((r & 0xff) ^ 0x80) - 0x80
    assert (r - lo) >> 8 == 128


@pytest.mark.parametrize("bits,K", [(64, 17), (256, 65), (512, 1001)])
def test_one_modulus_fewer_breaks_a_saturated_sum(bits, K):
    """Saturated sums (every significand all ones, every line's spread at the band width, all products of one
    sign: the sum sits just under the bound the count rule covers): the rule's modulus count reconstructs the
    exact sum and one modulus fewer does not (test_linalg.cpp:175-184, tight-modulus cases)."""
    n = bits // 32
    A = np.zeros((K, n + 3), np.uint32)
    A[:, :n] = 0xFFFFFFFF
    nb.set_fields(A, 0, 1)
    A[K - 1, n] = np.int32(-40).view(np.uint32)           # one low entry per line: spread 40
    exact = sum(aligned(A[k], -40, n) ** 2 for k in range(K))
    X, _, _ = model_dot(bits, A, A, K)
    assert X == exact
    X1, _, _ = model_dot(bits, A, A, K, drop=1)
    assert X1 != exact
