"""GPU: batched 4x4 complex LU (Engine::lu4, CommandBatch::lu4) against the C oracle, bit for bit.

The oracle restates the reference's rounding sequence (kernels.metal:210-249; pinned to MPFR replays
in test_oracle.py, as the reference's tests/test_batched4.cpp does).  Covered: every width class
from 64 to 1024 bits, composed and fused multiply-subtract, several right-hand sides, the inverse
and the determinant, singular systems that stop at each elimination step (status k + 1 and
division_by_zero solutions), pivots tied in magnitude (the lowest row wins), and 2,000 systems at
512 bits with one right-hand side, the configuration of the ragged benchmark."""
import numpy as np
import pytest

from limbforge_b200 import numbers as nb

pytestmark = pytest.mark.gpu


def systems(rng, bits, count, span=32):
    """count random systems [count * 16, 2, N+3] with singular and tied cases mixed in."""
    A = nb.random_complex(rng, count * 16, bits, span).reshape(count, 16, 2, -1)
    for m in range(0, count, 7):                 # column 0 zero: status 1
        A[m, 0::4] = 0
    for m in range(3, count, 11):                # rows 2 and 3 equal: rank 3, status 4
        A[m, 12:16] = A[m, 8:12]
    for m in range(5, count, 13):                # rows 0 and 1 equal: status 2
        A[m, 4:8] = A[m, 0:4]
    for m in range(6, count, 9):                 # |column 0| tied in magnitude on every row, signs differ
        v = A[m, 0, 0].copy()
        for r in range(4):
            A[m, 4 * r, 0] = v
            A[m, 4 * r, 1] = v
            if r & 1:
                A[m, 4 * r, 0] = nb.negate(v[None])[0]
    for m in range(2, count, 17):                # exact real pivots and zero imaginary parts
        A[m, :, 1] = 0
    return np.ascontiguousarray(A.reshape(count * 16, 2, -1))


@pytest.mark.parametrize("bits", [64, 128, 256, 416, 512, 1024])
@pytest.mark.parametrize("fused", [False, True])
def test_lu4_vs_oracle(engine, oracle, bits, fused):
    from limbforge_b200.api import Batched4
    rng = np.random.default_rng(bits * 3 + fused)
    count = 150
    A = systems(rng, bits, count)
    for rhs, inverse, det in ((1, False, True), (3, False, False), (0, True, True)):
        R = 4 if inverse else rhs
        B = nb.random_complex(rng, max(count * 4 * R, 1), bits, 32) if not inverse else None
        shape = Batched4(count=count, rhs=rhs, inverse=inverse, determinant=det, fused=fused)
        X, D, S, _ = engine.lu4(bits, shape, A, B)
        flags = int(fused) | (2 if det else 0) | (4 if inverse else 0)
        WX, WD, WS = oracle.lu4(bits, count, rhs, flags, A, B)
        assert (S == WS).all(), f"status rhs={rhs} inverse={inverse}"
        assert set(np.unique(WS)) >= {0, 1}, "the singular cases reach the kernel"
        bad = np.nonzero((X != WX).reshape(count, -1).any(axis=1))[0]
        assert bad.size == 0, f"X differs for systems {bad[:5]} rhs={rhs} inverse={inverse}"
        if det:
            assert (D == WD).all(), "determinant"


def test_lu4_512bit_2000_systems(engine, oracle):
    from limbforge_b200.api import Batched4
    rng = np.random.default_rng(512)
    count, bits = 2000, 512
    A = nb.random_complex(rng, count * 16, bits, 32)
    B = nb.random_complex(rng, count * 4, bits, 32)
    X, D, S, _ = engine.lu4(bits, Batched4(count=count, rhs=1, determinant=True), A, B)
    WX, WD, WS = oracle.lu4(bits, count, 1, 2, A, B)
    assert (S == WS).all() and (X == WX).all() and (D == WD).all()


def test_lu4_resident_batch_equals_host_call(engine, oracle):
    """CommandBatch::lu4 on buffers gives the host-array call's bits."""
    from limbforge_b200.api import Batched4
    rng = np.random.default_rng(77)
    bits, count = 256, 64
    A = systems(rng, bits, count)
    B = nb.random_complex(rng, count * 4 * 2, bits, 32)
    shape = Batched4(count=count, rhs=2, determinant=True, fused=True)
    bA, bB = engine.make_buffer(count * 16, bits, True), engine.make_buffer(count * 8, bits, True)
    bX, bD = engine.make_buffer(count * 8, bits, True), engine.make_buffer(count, bits, True)
    bS = engine.make_buffer(count)
    bA.upload(A)
    bB.upload(B)
    batch = engine.batch()
    batch.lu4(shape, bA, bB, bX, bD, bS)
    batch.submit().wait()
    WX, WD, WS = oracle.lu4(bits, count, 2, 3, A, B)
    assert (bX.download() == WX).all() and (bD.download() == WD).all()
    assert (bS.download().ravel() == WS).all()
