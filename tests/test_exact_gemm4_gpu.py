"""GPU: the exact batched 4 x 4 product (the reference's experimental ExactGemm4) against the oracle, bit for bit.

Every width from 64 to 1024 bits, real and complex, with and without accumulation and negation; random, cancelling
and wide-spread operands (spreads far beyond one cluster window, which the device streams); broadcast inputs
(stride 0), padded strides whose gaps stay untouched, statuses, empty sums; through the host-array call and a
resident batch whose ticket resolves after the wait, with a later operation in the same batch reading the output."""
import numpy as np
import pytest

from limbforge_b200 import api
from limbforge_b200 import numbers as nb
from test_exact_gemm4_oracle import operands

pytestmark = pytest.mark.gpu


def shape_dict(s: api.ExactGemm4Shape) -> dict:
    return {"count": s.count, "stride_a": s.stride_a, "stride_b": s.stride_b, "stride_c": s.stride_c,
            "accumulate": s.accumulate, "negative": s.negative}


@pytest.mark.parametrize("limbs", range(2, 33))
@pytest.mark.parametrize("cx", [False, True])
def test_exact_gemm4_every_width_vs_oracle(engine, oracle, limbs, cx):
    bits = 32 * limbs
    rng = np.random.default_rng(limbs * 2 + cx)
    g = api.ExactGemm4(engine)
    count = 40
    for span, accumulate, negative in ((6, False, False), (60, True, False), (5000, True, True)):
        A, B, Cm = (operands(bits, count, cx, rng, span) for _ in range(3))
        B[16:32] = A[16:32]
        if not cx:
            A[20:24] = nb.negate(A[16:20])                    # row 1 of matrix 1 cancels row 0
        s = api.ExactGemm4Shape(count, 16, 16, 16, accumulate, negative)
        want = oracle.exact_gemm4(bits, cx, shape_dict(s), A, B, Cm)
        got = Cm.copy()
        _, rep = g.gemm(bits, cx, s, A, B, got)
        bad = np.nonzero((got != want).reshape(count * 16, -1).any(axis=1))[0]
        assert bad.size == 0, f"span {span}: first differing components {bad[:5]}"
        assert rep.gpu_components == count * 16 * (2 if cx else 1) and rep.host_components == 0


@pytest.mark.parametrize("bits,cx", [(128, False), (320, True), (1024, False)])
def test_exact_gemm4_strides_broadcast_and_gaps(engine, oracle, bits, cx):
    rng = np.random.default_rng(bits + cx)
    g = api.ExactGemm4(engine)
    count = 25
    s = api.ExactGemm4Shape(count, 0, 19, 21, True, False)
    A = operands(bits, 1, cx, rng, 30)
    B = operands(bits, 2 * count, cx, rng, 30)[:19 * (count - 1) + 16]
    Cm = operands(bits, 2 * count, cx, rng, 30)[:21 * (count - 1) + 16]
    want = oracle.exact_gemm4(bits, cx, shape_dict(s), A, B, Cm)
    got = Cm.copy()
    g.gemm(bits, cx, s, A, B, got)
    assert (got == want).all()
    gaps = np.ones(len(Cm), bool)
    for t in range(count):
        gaps[21 * t:21 * t + 16] = False
    assert (got[gaps] == Cm[gaps]).all()                      # padding between output matrices untouched


@pytest.mark.parametrize("bits,cx,sa,accumulate", [(1024, True, 16, True), (1024, True, 0, False), (64, False, 16, True)])
def test_exact_gemm4_host_chunks(engine, oracle, bits, cx, sa, accumulate):
    """Host arrays run through the staged pipeline in several chunks (8 MiB of matrices per operand each)."""
    rng = np.random.default_rng(bits + sa + accumulate)
    g = api.ExactGemm4(engine)
    per = 16 * (bits // 8 + 12) * (2 if cx else 1)
    count = 2 * ((8 << 20) // per) + 37                        # two whole chunks and a ragged third
    s = api.ExactGemm4Shape(count, sa, 16, 16, accumulate, False)
    A = operands(bits, 1 if sa == 0 else count, cx, rng, 50)
    B, Cm = (operands(bits, count, cx, rng, 50) for _ in range(2))
    want = oracle.exact_gemm4(bits, cx, shape_dict(s), A, B, Cm)
    got = Cm.copy()
    t, rep = g.gemm(bits, cx, s, A, B, got)
    bad = np.nonzero((got != want).reshape(count * 16, -1).any(axis=1))[0]
    assert bad.size == 0, f"first differing components {bad[:5]}"
    assert rep.gpu_components == count * 16 * (2 if cx else 1) and t.gpu_seconds > 0


def test_exact_gemm4_statuses_and_empty_sums(engine, oracle):
    bits, w = 256, 11
    rng = np.random.default_rng(9)
    g = api.ExactGemm4(engine)
    A = nb.random_numbers(rng, 48, bits, 4)
    B = nb.random_numbers(rng, 48, bits, 4)
    Cm = nb.random_numbers(rng, 48, bits, 4)
    A[3, w - 1] = nb.INVALID
    B[16 + 5, w - 1] = nb.DIVISION_BY_ZERO
    Cm[40, w - 1] = nb.EXPONENT_OVERFLOW
    A[32:48] = 0
    for accumulate in (False, True):
        for negative in (False, True):
            s = api.ExactGemm4Shape(3, 16, 16, 16, accumulate, negative)
            want = oracle.exact_gemm4(bits, False, shape_dict(s), A, B, Cm)
            got = Cm.copy()
            g.gemm(bits, False, s, A, B, got)
            assert (got == want).all(), (accumulate, negative)
    assert (nb.status(want[0:4]) == nb.INVALID).all()


def test_exact_gemm4_resident_batch_ticket(engine, oracle):
    bits, cx, count = 512, True, 300
    rng = np.random.default_rng(5)
    g = api.ExactGemm4(engine)
    A, B, Cm = (operands(bits, count, cx, rng, 200) for _ in range(3))
    s = api.ExactGemm4Shape(count, 16, 16, 16, True, True)
    want = oracle.exact_gemm4(bits, cx, shape_dict(s), A, B, Cm)
    bufs = [engine.make_buffer(count * 16, bits, cx) for _ in range(4)]
    for buf, x in zip(bufs, (A, B, Cm)):
        buf.upload(x)
    batch = engine.batch()
    ticket = g.encode(batch, s, bufs[0], bufs[1], bufs[2])
    batch.run(api.Operation.complex_add, bufs[2], bufs[2], bufs[3])   # reads the product later in the same batch
    assert not ticket.resolved()
    with pytest.raises(api.LogicError):
        ticket.report()
    sub = batch.submit()
    sub.wait()
    assert ticket.resolved()
    rep = ticket.report()
    assert rep.gpu_components == count * 32 and rep.host_components == 0 and not rep.provisional_reads
    assert (bufs[2].download() == want).all()
    assert (bufs[3].download() == oracle.elementwise(bits, int(api.Operation.complex_add), want, want)).all()


def test_exact_gemm4_overlapping_inputs(engine, oracle):
    bits = 192
    rng = np.random.default_rng(11)
    g = api.ExactGemm4(engine)
    s = api.ExactGemm4Shape(30, 4, 1, 16, False, True)         # input matrices overlap, as the reference allows
    A = nb.random_numbers(rng, 4 * 29 + 16, bits, 20)
    B = nb.random_numbers(rng, 29 + 16, bits, 20)
    Cm = nb.random_numbers(rng, 16 * 30, bits, 20)
    want = oracle.exact_gemm4(bits, False, shape_dict(s), A, B, Cm)
    got = Cm.copy()
    g.gemm(bits, False, s, A, B, got)
    assert (got == want).all()


def test_exact_gemm4_argument_errors(engine):
    g = api.ExactGemm4(engine)
    x = np.zeros((32, 5), np.uint32)
    with pytest.raises(api.InvalidArgument):
        g.gemm(64, False, api.ExactGemm4Shape(2, 16, 16, 8), x, x, x.copy())      # overlapping outputs
    with pytest.raises(api.InvalidArgument):
        g.gemm(48, False, api.ExactGemm4Shape(1), x, x, x.copy())                 # not a whole number of limbs
    t, rep = g.gemm(64, False, api.ExactGemm4Shape(0), x, x, x.copy())
    assert rep.gpu_components == 0
