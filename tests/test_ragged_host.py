"""CPU: host-side layout of ragged mixed-precision batches (lf_ragged_pack) through the C ABI.

Packing is pure host code: every instance gets A, B and C in turn at 256-byte aligned offsets,
then the LU job's operands; sizes follow the element layout (bits/8 + 12 bytes, doubled for
complex) and invalid precisions are rejected."""
import numpy as np
import pytest

from limbforge_b200 import api
from limbforge_b200.numbers import element_bytes


def test_pack_offsets_are_aligned_and_disjoint():
    rng = np.random.default_rng(3)
    count = 200
    bits = rng.choice([64, 96, 128, 256, 512, 1024], size=count)
    m, n, k = (rng.integers(0, 12, size=count) for _ in range(3))
    items = api.ragged_items(bits, m, n, k)
    lu = api.RaggedLu4(512, api.Batched4(count=10, rhs=2, determinant=True))
    total = api.ragged_pack(True, items, lu)
    spans = []
    for it in items:
        es = element_bytes(int(it["bits"]), True)
        for off, elems in ((it["a"], it["m"] * it["k"]), (it["b"], it["k"] * it["n"]), (it["c"], it["m"] * it["n"])):
            assert off % 256 == 0
            spans.append((int(off), int(off) + int(elems) * es))
    ces = element_bytes(512, True)
    for off, size in ((lu.A, 10 * 16 * ces), (lu.B, 10 * 4 * 2 * ces), (lu.X, 10 * 4 * 2 * ces), (lu.det, 10 * ces),
                      (lu.status, 10 * 4)):
        assert off % 256 == 0
        spans.append((off, off + size))
    spans.sort()
    for (a0, a1), (b0, b1) in zip(spans, spans[1:]):
        assert a1 <= b0
    assert spans[-1][1] <= total < spans[-1][1] + 256


def test_pack_real_elements_are_half_size():
    items = api.ragged_items([256, 256], [3, 5], [4, 2], [7, 1])
    total_c = api.ragged_pack(True, items.copy())
    total_r = api.ragged_pack(False, items)
    assert items["b"][0] - items["a"][0] == ((3 * 7 * element_bytes(256) + 255) // 256) * 256
    assert total_r < total_c


@pytest.mark.parametrize("bits", [32, 48, 1056, 0])
def test_pack_rejects_bad_precisions(bits):
    items = api.ragged_items([256, bits], [2, 2], [2, 2], [2, 2])
    with pytest.raises(api.InvalidArgument):
        api.ragged_pack(True, items)


def test_pack_rejects_an_lu_job_with_inverse_and_rhs():
    items = api.ragged_items([128], [2], [2], [2])
    with pytest.raises(api.InvalidArgument):
        api.ragged_pack(True, items, api.RaggedLu4(512, api.Batched4(count=4, rhs=1, inverse=True)))
