"""GPU: complex fused multiply-add and multiply-subtract (each component one rounding of
a*b + c*d + e) on operands that reach every branch of the three-term exact sum
(tests/fused_cases.py: exact and near cancellation, straddling and far terms, ties, range
limits), against the C oracle bit for bit at widths from 64 to 1024 bits, and through the fused
strided GEMM, whose every step is such a sum."""
import numpy as np
import pytest

from fused_cases import dot2_cases
from limbforge_b200 import numbers as nb

pytestmark = pytest.mark.gpu

WIDTHS = [64, 96, 128, 256, 352, 512, 768, 1024]


@pytest.mark.parametrize("bits", WIDTHS)
def test_cfma_three_term_cases(engine, oracle, bits):
    from limbforge_b200.api import Operation
    rng = np.random.default_rng(900 + bits)
    a, b, c = dot2_cases(rng, bits, 640)
    for op in (11, 12):
        got = engine.run_ternary(bits, Operation(op), a, b, c)[0]
        want = oracle.elementwise(bits, op, a, b, c)
        bad = np.nonzero((got != want).reshape(got.shape[0], -1).any(axis=1))[0]
        assert bad.size == 0, f"op {op}: cases {bad[:8]} (kinds {bad[:8] % 8})"


@pytest.mark.parametrize("bits", [128, 512])
def test_fused_strided_gemm_with_cancelling_steps(engine, oracle, bits):
    """C (+)= A B with fused complex steps, C starting at -RN(A B): the last steps cancel deeply."""
    from limbforge_b200.api import BatchedLinalg, StridedGemm
    rng = np.random.default_rng(31 + bits)
    count, m, n, k = 12, 5, 4, 9
    A = nb.random_complex(rng, count * m * k, bits, 20)
    B = nb.random_complex(rng, count * k * n, bits, 20)
    shape = {"count": count, "m": m, "n": n, "k": k, "stride_a": m * k, "stride_b": k * n, "stride_c": m * n, "fused": True}
    P = oracle.strided_gemm(bits, True, shape, A, B, np.zeros((count * m * n, 2, bits // 32 + 3), np.uint32))
    C = np.ascontiguousarray(np.stack([nb.negate(P[:, 0]), nb.negate(P[:, 1])], axis=1))
    s = StridedGemm(count=count, m=m, n=n, k=k, stride_a=m * k, stride_b=k * n, stride_c=m * n, accumulate=True, fused=True)
    got = C.copy()
    BatchedLinalg(engine).gemm(bits, True, s, A, B, got)
    want = oracle.strided_gemm(bits, True, dict(shape, accumulate=True), A, B, C)
    assert (got == want).all()
