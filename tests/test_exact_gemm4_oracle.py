"""CPU: pin the oracle's exact batched 4 x 4 product (lf_oracle.c lfo_exact_gemm4, the contract of the reference's
benchmarks/experiments/exact_gemm4: one rounding of C_old + the exact products per component, optional negation,
broadcasts by stride 0) against independent MPFR sums (mpfr_sum over the same exact products) on random, cancelling,
tie and wide-spread inputs, real and complex; and its status and empty-sum rules."""
import numpy as np
import pytest

from limbforge_b200 import numbers as nb
from oracle.oracle import Mpfr


def operands(bits, count, cx, rng, span):
    w = bits // 32 + 3
    shape = (count * 16, 2, w) if cx else (count * 16, w)
    x = np.zeros(shape, np.uint32)
    if cx:
        x[:, 0] = nb.random_numbers(rng, count * 16, bits, span, zero_frac=0.05, sparse_frac=0.1)
        x[:, 1] = nb.random_numbers(rng, count * 16, bits, span, zero_frac=0.05, sparse_frac=0.1)
    else:
        x[:] = nb.random_numbers(rng, count * 16, bits, span, zero_frac=0.05, sparse_frac=0.1)
    return x


@pytest.mark.parametrize("bits", [64, 352, 1024])
@pytest.mark.parametrize("cx", [False, True])
def test_exact_gemm4_oracle_vs_mpfr(oracle, bits, cx):
    mp = Mpfr()
    rng = np.random.default_rng(bits + 7 * cx)
    count = 6
    for span, accumulate, negative in ((6, False, False), (40, True, False), (3000, True, True), (6, False, True)):
        A, B, C = (operands(bits, count, cx, rng, span) for _ in range(3))
        B[16:32] = A[16:32]                                   # matrix 1: B = A, and a row cancelling another
        A[20:24] = nb.negate(A[16:20].reshape(-1, bits // 32 + 3)).reshape(A[20:24].shape) if not cx else A[20:24]
        shape = {"count": count, "stride_a": 16, "stride_b": 16, "stride_c": 16, "accumulate": accumulate, "negative": negative}
        got = oracle.exact_gemm4(bits, cx, shape, A, B, C)
        for t in range(count):
            for i in range(4):
                for j in range(4):
                    o = t * 16 + i * 4 + j
                    if not cx:
                        a = np.ascontiguousarray(A[t * 16 + i * 4:t * 16 + i * 4 + 4])
                        b = np.ascontiguousarray(B[t * 16 + j::4][:4])
                        want = mp.dot(bits, C[o] if accumulate else None, False, a, 1, b, 1, 4)
                        if negative:
                            want = nb.negate(want[None])[0]
                        assert (got[o] == want).all(), (span, t, i, j)
                    else:
                        a = np.ascontiguousarray(A[t * 16 + i * 4:t * 16 + i * 4 + 4].reshape(8, -1))
                        bz = B[t * 16 + j::4][:4]
                        br = np.ascontiguousarray(np.stack([bz[:, 0], nb.negate(bz[:, 1])], 1).reshape(8, -1))
                        bi = np.ascontiguousarray(np.stack([bz[:, 1], bz[:, 0]], 1).reshape(8, -1))
                        for part, bb in ((0, br), (1, bi)):
                            want = mp.dot(bits, np.ascontiguousarray(C[o, part]) if accumulate else None, False, a, 1, bb, 1, 8)
                            if negative:
                                want = nb.negate(want[None])[0]
                            assert (got[o, part] == want).all(), (span, t, i, j, part)


def test_exact_gemm4_oracle_rules(oracle):
    bits = 256
    w = bits // 32 + 3
    rng = np.random.default_rng(3)
    A = nb.random_numbers(rng, 32, bits, 4)
    B = nb.random_numbers(rng, 16, bits, 4)
    C = nb.random_numbers(rng, 32, bits, 4)
    A[3, w - 1] = nb.INVALID                                  # row 0 of matrix 0 reads it: outputs 0..3 carry it
    shape = {"count": 2, "stride_a": 16, "stride_b": 0, "stride_c": 16, "accumulate": True, "negative": False}
    got = oracle.exact_gemm4(bits, False, shape, A, B, C)
    assert (nb.status(got[0:4]) == nb.INVALID).all() and (nb.sign(got[0:4]) == 0).all()
    assert (nb.status(got[4:]) == 0).all()
    # no nonzero product: the old value itself; without accumulation, zero
    Z = np.zeros_like(A)
    assert (oracle.exact_gemm4(bits, False, shape, Z, B, C) == C).all()
    shape["accumulate"] = False
    assert (oracle.exact_gemm4(bits, False, shape, Z, B, C) == 0).all()
    # broadcast B (stride 0): both matrices use the same B
    g2 = oracle.exact_gemm4(bits, False, shape, np.concatenate([A[16:], A[16:]]), B, C)
    assert (g2[:16] == g2[16:]).all()
