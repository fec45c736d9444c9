"""CPU: the oracle's precision cast and tree sum, pinned before any GPU result is compared with them.

cast is checked against MPFR (mpfr_set into the target precision, round to nearest even) on random
values, exact ties, values one unit from a power of two, zeros, statuses and the exponent limits.
tree_sum is checked against the reference's own add and cadd (core.hpp, compiled into oracle/_ref)
applied level by level in the adjacent-pair order of the reference's tree kernels."""
import numpy as np
import pytest

from limbforge_b200 import numbers as nb
from oracle.oracle import Mpfr, Oracle, Reference


@pytest.fixture(scope="module")
def orc():
    return Oracle()


def cast_cases(rng, bits, cnt=600):
    x = nb.random_numbers(rng, cnt, bits, 1000, zero_frac=0.05, sparse_frac=0.1)
    n = bits // 32
    q = cnt // 6
    x[:q, :n] = 0xFFFFFFFF                      # all ones: rounding up carries into a new binade
    x[q:2 * q, :n - 1] = 0
    x[q:2 * q, 0] = rng.integers(0, 4, size=q)  # few bits below the top: ties and exact casts
    x[2 * q:3 * q, n] = np.int32(1_000_000_000).view(np.uint32)      # at the exponent limit
    x[3 * q:3 * q + 10, n + 2] = 4                                    # statuses pass through
    x[3 * q + 10:3 * q + 20, n + 2] = 2
    return x


@pytest.mark.parametrize("from_bits,to_bits", [(64, 1024), (256, 128), (1024, 64), (512, 512), (96, 64), (800, 224), (128, 96)])
def test_cast_matches_mpfr(orc, from_bits, to_bits):
    rng = np.random.default_rng(from_bits * 7 + to_bits)
    x = cast_cases(rng, from_bits)
    got = orc.cast(from_bits, to_bits, False, x)
    want = Mpfr().cast(from_bits, to_bits, x)
    bad = np.nonzero((got != want).any(axis=1))[0]
    assert bad.size == 0, f"first differing element {bad[:5]}"


def test_cast_complex_is_componentwise(orc):
    rng = np.random.default_rng(4)
    z = nb.random_complex(rng, 200, 512, 100)
    got = orc.cast(512, 160, True, z)
    assert (got[:, 0] == orc.cast(512, 160, False, np.ascontiguousarray(z[:, 0]))).all()
    assert (got[:, 1] == orc.cast(512, 160, False, np.ascontiguousarray(z[:, 1]))).all()


@pytest.mark.skipif(not Reference.available(), reason="reference build absent")
@pytest.mark.parametrize("bits,complex_", [(64, False), (256, False), (1024, False), (128, True), (512, True)])
def test_tree_sum_matches_reference_adds(orc, bits, complex_):
    ref = Reference()
    rng = np.random.default_rng(bits + complex_)
    for count in (0, 1, 2, 3, 5, 8, 13, 64, 257):
        x = (nb.random_complex(rng, count, bits, 60, zero_frac=0.05) if complex_ else
             nb.random_numbers(rng, count, bits, 60, zero_frac=0.05))
        if count > 4:
            x[1] = nb.negate(x[0:1])[0]         # exact cancellation inside the tree
        cur = x.copy()
        while cur.shape[0] > 1:
            pairs = cur.shape[0] // 2
            s = ref.elementwise(bits, 4 if complex_ else 0, np.ascontiguousarray(cur[0:2 * pairs:2]),
                                np.ascontiguousarray(cur[1:2 * pairs:2]))
            cur = np.concatenate([s, cur[2 * pairs:]]) if cur.shape[0] % 2 else s
        want = cur[0] if count else np.zeros_like(orc.tree_sum(bits, complex_, x))
        assert (orc.tree_sum(bits, complex_, x) == want).all(), f"count={count}"
