"""GPU: precision casts and tree sums against the oracle, bit for bit.

Casts run between every pair of a spread of widths in both directions (exact widening, RNE
narrowing), over random values, ties, all-ones significands that round into the next binade, the
exponent limit, zeros and statuses, real and complex; through the host-array call, a resident batch
and the device-pointer entry.  Tree sums follow the reference's adjacent-pair tree over counts from 0
to 65,537, real and complex, with an exact cancellation inside the tree."""
import numpy as np
import pytest

from limbforge_b200 import api
from limbforge_b200 import numbers as nb
from test_oracle_cast_tree import cast_cases

pytestmark = pytest.mark.gpu

WIDTHS = [64, 96, 128, 256, 512, 800, 1024]


@pytest.mark.parametrize("from_bits", WIDTHS)
def test_cast_every_pair_vs_oracle(engine, oracle, from_bits):
    rng = np.random.default_rng(from_bits)
    x = cast_cases(rng, from_bits, 480)
    for to_bits in WIDTHS:
        got, _ = engine.cast(from_bits, to_bits, False, x)
        want = oracle.cast(from_bits, to_bits, False, x)
        bad = np.nonzero((got != want).any(axis=1))[0]
        assert bad.size == 0, f"{from_bits}->{to_bits}: first differing element {bad[:5]}"


def test_cast_complex_resident_and_device_pointer(engine, oracle):
    import torch
    rng = np.random.default_rng(3)
    z = nb.random_complex(rng, 1000, 768, 200, zero_frac=0.02)
    want = oracle.cast(768, 192, True, z)
    a = engine.make_buffer(1000, 768, True)
    o = engine.make_buffer(1000, 192, True)
    a.upload(z)
    b = engine.batch()
    b.cast(a, o)
    b.submit().wait()
    assert (o.download() == want).all()
    dz = torch.from_numpy(z.view(np.int32)).cuda()
    do = torch.zeros(want.size, dtype=torch.int32, device="cuda")
    api.dev_cast(768, 192, True, dz.data_ptr(), do.data_ptr(), 1000)
    torch.cuda.synchronize()
    assert (do.cpu().numpy().view(np.uint32).reshape(want.shape) == want).all()


@pytest.mark.parametrize("bits,complex_", [(64, False), (256, False), (1024, False), (128, True), (512, True)])
def test_tree_sum_vs_oracle(engine, oracle, bits, complex_):
    rng = np.random.default_rng(bits * 3 + complex_)
    for count in (0, 1, 2, 3, 5, 64, 1000, 65537):
        x = (nb.random_complex(rng, count, bits, 60, zero_frac=0.02) if complex_ else
             nb.random_numbers(rng, count, bits, 60, zero_frac=0.02))
        if count > 4:
            x[3] = nb.negate(x[2:3])[0]                 # exact cancellation inside the tree
        a = engine.make_buffer(count, bits, complex_)
        if count:
            a.upload(x)
        o = engine.make_buffer(1, bits, complex_)
        o.upload(nb.random_complex(rng, 1, bits, 5) if complex_ else nb.random_numbers(rng, 1, bits, 5))   # overwritten
        b = engine.batch()
        b.tree_sum(a, o)
        b.submit().wait()
        assert (o.download()[0] == oracle.tree_sum(bits, complex_, x)).all(), f"count={count}"


def test_tree_sum_device_pointer(oracle):
    import torch
    rng = np.random.default_rng(11)
    bits, count = 384, 4099
    x = nb.random_numbers(rng, count, bits, 30)
    dx = torch.from_numpy(x.view(np.int32)).cuda()
    out = torch.zeros(bits // 32 + 3, dtype=torch.int32, device="cuda")
    scratch = torch.zeros(2 * ((count + 1) // 2) * (bits // 32 + 3), dtype=torch.int32, device="cuda")
    api.dev_tree_sum(bits, False, dx.data_ptr(), count, out.data_ptr(), scratch.data_ptr())
    torch.cuda.synchronize()
    assert (out.cpu().numpy().view(np.uint32) == oracle.tree_sum(bits, False, x)).all()
