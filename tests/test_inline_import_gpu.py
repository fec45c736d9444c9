"""GPU: BatchedLinalg::import_inline_complex gathers complex values from MPFR significands inside one page-aligned host
allocation.  Significands are laid out as MPFR keeps them (ceil(N/2) little-endian 64-bit limbs, an odd width leaving
one low padding word), scattered over the allocation; records carry exponents, signs and statuses, including zeros,
statuses and exponents beyond the element range; every width from 64 to 1024 bits; and the argument checks."""
import numpy as np
import pytest

from limbforge_b200 import api
from limbforge_b200 import numbers as nb

pytestmark = pytest.mark.gpu


def stage(bits, values, rng):
    """Allocation + records for complex values (count, 2, N+3); returns (allocation, records, expected)."""
    n = bits // 32
    span = 8 * ((bits + 63) // 64)
    count = len(values)
    slots = rng.permutation(2 * count + 7)[:2 * count]            # scattered, not in element order
    alloc = api.page_aligned((2 * count + 7) * span + 64)
    rec = np.zeros(count, api.INLINE_RECORD_DTYPE)
    expect = values.copy()
    for i in range(count):
        for part, name in ((0, "real"), (1, "imag")):
            v = values[i, part]
            off = 64 + int(slots[2 * i + part]) * span
            words = alloc[off:off + span].view(np.uint32)
            words[n % 2:n % 2 + n] = v[:n]
            rec[f"{name}_offset"][i] = off
            rec[f"{name}_exponent"][i] = np.int32(v[n].view(np.int32))
            rec[f"{name}_sign"][i] = np.int32(v[n + 1].view(np.int32))
            rec[f"{name}_status"][i] = v[n + 2]
    return alloc, rec, expect


@pytest.mark.parametrize("limbs", range(2, 33))
def test_inline_import_every_width(engine, limbs):
    bits = 32 * limbs
    n = limbs
    rng = np.random.default_rng(limbs)
    count = 500
    values = nb.random_complex(rng, count, bits, 2000, zero_frac=0.05)
    values[7, 0, n + 2] = nb.INVALID                                 # a status: zero with that status
    values[7, 0, :n + 2] = 0
    alloc, rec, expect = stage(bits, values, rng)
    rec["imag_exponent"][9] = 1000000001                             # beyond the element range: exponent_overflow
    rec["imag_sign"][9] = 1
    expect[9, 1] = 0
    expect[9, 1, n + 2] = nb.EXPONENT_OVERFLOW
    out = engine.make_buffer(count, bits, True)
    bl = api.BatchedLinalg(engine)
    b = engine.batch()
    bl.import_inline_complex(b, alloc, rec, out)
    b.submit().wait()
    got = out.download()
    bad = np.nonzero((got != expect).reshape(count, -1).any(axis=1))[0]
    assert bad.size == 0, f"first differing elements {bad[:5]}"


def test_inline_import_argument_checks(engine):
    bits = 96
    rng = np.random.default_rng(1)
    values = nb.random_complex(rng, 4, bits, 10)
    alloc, rec, _ = stage(bits, values, rng)
    out = engine.make_buffer(4, bits, True)
    bl = api.BatchedLinalg(engine)
    bad = rec.copy()
    bad["real_offset"][2] += 4                                       # not on a 64-bit limb
    with pytest.raises(api.InvalidArgument):
        bl.import_inline_complex(engine.batch(), alloc, bad, out)
    bad = rec.copy()
    bad["imag_offset"][0] = alloc.nbytes - 8                         # runs past the allocation
    with pytest.raises(api.InvalidArgument):
        bl.import_inline_complex(engine.batch(), alloc, bad, out)
    with pytest.raises(api.InvalidArgument):                          # not whole pages
        bl.import_inline_complex(engine.batch(), alloc[8:], rec, out)
    with pytest.raises(api.InvalidArgument):
        bl.import_inline_complex(engine.batch(), alloc, rec, engine.make_buffer(4, bits, False))
