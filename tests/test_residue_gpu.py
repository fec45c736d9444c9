"""GPU: the int8-residue/CRT tensor-core engine (tcgen05 kind::i8) forced on shapes that are not
multiples of the 128 x 128 x 128 tiles, at several widths, for GEMM, SYRK and updates: bit-identical
to the generic limb kernel and to the oracle."""
import numpy as np
import pytest

from limbforge_b200 import numbers as nb

pytestmark = pytest.mark.gpu


def same(x, y):
    return x.shape == y.shape and bool((x == y).all())


@pytest.fixture(scope="module")
def engines(engine):
    from limbforge_b200 import api
    return api.Linalg(engine, api.LinalgOptions(method=2)), api.Linalg(engine, api.LinalgOptions(method=1))


@pytest.mark.parametrize("bits,m,n,k,span", [(64, 5, 3, 7, 4), (128, 130, 129, 200, 30), (256, 64, 200, 129, 40),
                                             (512, 257, 131, 300, 40), (1024, 40, 37, 65, 20), (96, 1, 1, 1, 0)])
def test_residue_gemm_matches_limb_and_oracle(engines, oracle, bits, m, n, k, span):
    res, limb = engines
    rng = np.random.default_rng(bits + m)
    A = nb.random_numbers(rng, k * m, bits, span, zero_frac=0.01, sparse_frac=0.05)
    B = nb.random_numbers(rng, k * n, bits, span, zero_frac=0.01, sparse_frac=0.05)
    C0 = nb.random_numbers(rng, m * n, bits, span + 10)
    for sub in (False, True):
        a, b = C0.copy(), C0.copy()
        res.gemm(bits, True, A, B, m, n, k, a, subtract=sub)
        r = res.report()
        assert r["method"] == 2 and r["moduli"] > 0
        limb.gemm(bits, True, A, B, m, n, k, b, subtract=sub)
        assert same(a, b), f"residue vs limb sub={sub}"
    rows = (0, min(m, 3))
    want = oracle.gemm(bits, True, A, B, m, n, k, C=C0, subtract=True, rows=rows)
    assert same(a[: rows[1] * n], want[: rows[1] * n])


@pytest.mark.parametrize("bits,rows,cols", [(128, 150, 70), (512, 129, 140)])
def test_residue_syrk_and_update(engines, oracle, bits, rows, cols):
    res, limb = engines
    rng = np.random.default_rng(rows)
    A = nb.random_numbers(rng, rows * cols, bits, 30, zero_frac=0.02)
    for lower in (True, False):
        a = np.zeros((cols * cols, bits // 32 + 3), np.uint32)
        b = a.copy()
        res.syrk(bits, A, rows, cols, a, lower_only=lower)
        limb.syrk(bits, A, rows, cols, b, lower_only=lower)
        assert same(a, b)
    C0 = nb.random_numbers(rng, cols * cols, bits, 40)
    a, b = C0.copy(), C0.copy()
    res.syrk(bits, A, rows, cols, a, lower_only=True, subtract=True)
    limb.syrk(bits, A, rows, cols, b, lower_only=True, subtract=True)
    assert same(a, b)
    want = oracle.syrk(bits, A, rows, cols, C=C0, lower_only=True, subtract=True, lines=(0, 4))
    assert same(a[: 4 * cols], want[: 4 * cols])


def test_residue_refuses_wide_lines(engines):
    from limbforge_b200.api import RuntimeFailure
    res, _ = engines
    bits = 128
    rng = np.random.default_rng(1)
    A = nb.random_numbers(rng, 16, bits, 4)
    A[3, bits // 32] = np.int32(5000).view(np.uint32)            # a line spanning more than 192 bits
    C = np.zeros((16, bits // 32 + 3), np.uint32)
    with pytest.raises(RuntimeFailure):
        res.gemm(bits, False, A, A, 4, 4, 4, C)
