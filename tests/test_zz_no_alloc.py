"""GPU: the allocation-free exact product (lf_dev_exact_product_static).

Callers that cannot allocate device memory when they need a product (a fixed device-memory plan,
threads that must not take the allocator's locks, runtimes that forbid allocation) use this entry
point; it keeps its temporaries in a static 32 MiB device array of the library.  Here it is called
through the C ABI and must give exactly the bits of the allocating entry point
(lf_dev_exact_product) on two calls in a row with different shapes, widths and modes (the array keeps
the previous call's contents), and reject a product whose scratch would not fit.  This file is
collected last so that a failure here does not stop the rest of the suite."""
import ctypes as C

import numpy as np
import pytest

from limbforge_b200 import numbers as nb

pytestmark = pytest.mark.gpu


def _entry(lib, name):
    f = getattr(lib, name)
    V, S, I = C.c_void_p, C.c_size_t, C.c_int
    f.argtypes = [I, V, S, S, V, S, S, S, S, S, V, S, I, I, V] if name.endswith("static") else \
        [V, I, V, S, S, V, S, S, S, S, S, V, S, I, I, V]
    f.restype = I
    return f


def _product(api, la, static, bits, A, B, m, n, k, C0, subtract, lower, transpose_rows):
    """C <- RN(C0 -/+ op(A) B) on device buffers; A is k x m (transposed) or m x k."""
    eng = la.engine
    bufs = [eng.make_buffer(x.shape[0], bits) for x in (A, B, C0)]
    for b, x in zip(bufs, (A, B, C0)):
        b.upload(x)
    pa, pb, pc = (b.device_pointer() for b in bufs)
    lv = (1, m) if transpose_rows else (k, 1)                 # left line i: column i of A, or row i
    rv = (1, n)                                               # right line j: column j of B
    if static:
        f = _entry(api.lib, "lf_dev_exact_product_static")
        rc = f(bits, pa, lv[0], lv[1], pb, rv[0], rv[1], m, n, k, pc, n, int(subtract), int(lower), None)
    else:
        f = _entry(api.lib, "lf_dev_exact_product")
        rc = f(la.handle, bits, pa, lv[0], lv[1], pb, rv[0], rv[1], m, n, k, pc, n, int(subtract), int(lower), None)
    api.check(rc)
    return bufs[2].download()


def test_static_scratch_product_matches_allocating_entry_point():
    from limbforge_b200 import api
    eng = api.Engine()
    la = api.Linalg(eng)
    rng = np.random.default_rng(2026)
    cases = [(512, 100, 90, 130, True, False), (256, 64, 64, 80, False, True)]   # two calls in a row
    for bits, m, n, k, subtract, lower in cases:
        A = nb.random_numbers(rng, k * m, bits, 40, zero_frac=0.01)
        B = nb.random_numbers(rng, k * n, bits, 40, zero_frac=0.01)
        C0 = nb.random_numbers(rng, m * n, bits, 50)
        got = _product(api, la, True, bits, A, B, m, n, k, C0, subtract, lower, True)
        want = _product(api, la, False, bits, A, B, m, n, k, C0, subtract, lower, True)
        assert (got == want).all(), f"bits={bits} m={m} n={n} k={k}"


def test_static_scratch_product_rejects_oversized_problems():
    from limbforge_b200 import api
    eng = api.Engine()
    la = api.Linalg(eng)
    bits, m, n, k = 1024, 2000, 2000, 8        # residues alone need far more than the static area
    rng = np.random.default_rng(7)
    A = nb.random_numbers(rng, k * m, bits, 4)
    B = nb.random_numbers(rng, k * n, bits, 4)
    C0 = np.zeros((m * n, bits // 32 + 3), np.uint32)
    with pytest.raises(api.InvalidArgument, match="static area"):
        _product(api, la, True, bits, A, B, m, n, k, C0, False, False, True)
