"""GPU: segmented dot products (Engine::segmented_dot, CommandBatch::segmented_dot) and four-term complex
recurrences (Engine::recurrence) against the C oracle, bit for bit; the oracle is pinned to the reference's
own fma / cfma / cmul / cadd in test_oracle.py.  Real and complex chains, per-segment and shared right
operands, empty segments and zero-length chains, recurrences with zero and several steps and shared weights."""
import numpy as np
import pytest

from limbforge_b200 import numbers as nb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bits", [64, 192, 512, 1024])
@pytest.mark.parametrize("complex_", [False, True])
def test_segmented_dot_vs_oracle(engine, oracle, bits, complex_):
    from limbforge_b200.api import SegmentedDot
    rng = np.random.default_rng(bits + 10 * complex_)
    make = (lambda c: nb.random_complex(rng, c, bits, 40, zero_frac=0.02)) if complex_ else \
        (lambda c: nb.random_numbers(rng, c, bits, 40, zero_frac=0.02, sparse_frac=0.05))
    for seg, ln, shared in ((300, 17, False), (257, 6, True), (5, 0, False), (0, 4, True)):
        a = make(max(seg * ln, 1))
        b = make(max(ln if shared else seg * ln, 1))
        got, _ = engine.segmented_dot(bits, complex_, SegmentedDot(seg, ln, shared), a, b)
        want = oracle.segmented_dot(bits, complex_, seg, ln, shared, a, b)
        assert (got == want).all(), f"segments={seg} length={ln} shared={shared}"


def test_segmented_dot_resident_batch(engine, oracle):
    from limbforge_b200.api import SegmentedDot
    bits, seg, ln = 320, 64, 11
    rng = np.random.default_rng(5)
    a, b = nb.random_complex(rng, seg * ln, bits, 30), nb.random_complex(rng, seg * ln, bits, 30)
    A, B, O = engine.make_buffer(seg * ln, bits, True), engine.make_buffer(seg * ln, bits, True), engine.make_buffer(seg, bits, True)
    A.upload(a)
    B.upload(b)
    batch = engine.batch()
    batch.segmented_dot(SegmentedDot(seg, ln, False), A, B, O)
    batch.submit().wait()
    assert (O.download() == oracle.segmented_dot(bits, True, seg, ln, False, a, b)).all()


@pytest.mark.parametrize("bits", [128, 256, 768])
def test_recurrence_vs_oracle(engine, oracle, bits):
    rng = np.random.default_rng(bits + 3)
    for count, steps, spw in ((500, 9, 1), (96, 4, 4), (33, 0, 1)):
        seeds = nb.random_complex(rng, 4 * count, bits, 4)
        weights = nb.random_complex(rng, max(steps * 4 * (count // spw), 1), bits, 2)
        got, _ = engine.recurrence(bits, seeds, weights, count, steps, spw)
        want = oracle.recurrence(bits, seeds, weights, count, steps, spw)
        assert (got == want).all(), f"count={count} steps={steps} spw={spw}"
