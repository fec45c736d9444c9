"""GPU: the allocation-free exact product (lf_dev_exact_product_static).

Callers that cannot allocate device memory when they need a product (a fixed device-memory plan,
threads that must not take the allocator's locks, runtimes that forbid allocation) use this entry
point; it keeps its temporaries in a static 32 MiB device array of the library.  Here it is called
through the C ABI and must give exactly the bits of the allocating entry point
(lf_dev_exact_product) on calls in a row with different shapes, widths and modes (the array keeps
the previous call's contents), reuse its modulus tables for the same width, take the limb kernel
both for wide bands and for products whose planes do not fit the array, allocate no device memory
once warm, and reject a product with more lines than its line table holds.  This file is collected
last so that a failure here does not stop the rest of the suite."""
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


def _buffers(eng, bits, *arrays):
    bufs = [eng.make_buffer(x.shape[0], bits) for x in arrays]
    for b, x in zip(bufs, arrays):
        b.upload(x)
    return bufs


def _call(api, la, static, bits, bufs, m, n, k, subtract, lower):
    """C <- RN(C -/+ A^T B) (A is k x m, B is k x n) on device buffers, through the C ABI."""
    pa, pb, pc = (b.device_pointer() for b in bufs)
    if static:
        rc = _entry(api.lib, "lf_dev_exact_product_static")(bits, pa, 1, m, pb, 1, n, m, n, k, pc, n, int(subtract), int(lower), None)
    else:
        rc = _entry(api.lib, "lf_dev_exact_product")(la.handle, bits, pa, 1, m, pb, 1, n, m, n, k, pc, n, int(subtract), int(lower), None)
    api.check(rc)


def _product(api, la, static, bits, A, B, m, n, k, C0, subtract, lower):
    bufs = _buffers(la.engine, bits, A, B, C0)
    _call(api, la, static, bits, bufs, m, n, k, subtract, lower)
    return bufs[2].download()


def test_static_scratch_product_matches_allocating_entry_point():
    from limbforge_b200 import api
    eng = api.Engine()
    la = api.Linalg(eng)
    rng = np.random.default_rng(2026)
    # calls in a row: a new width each time, then the same width twice (cached modulus tables), a
    # 1024-bit product, a band wider than the residue engine takes (limb kernel) and K = 0
    cases = [(512, 100, 90, 130, 40, True, False), (256, 64, 64, 80, 40, False, True), (256, 70, 33, 96, 30, True, False),
             (1024, 40, 50, 64, 20, True, False), (512, 48, 40, 56, 400, True, False), (384, 20, 30, 0, 10, True, False)]
    for bits, m, n, k, spread, subtract, lower in cases:
        A = nb.random_numbers(rng, k * m, bits, spread, zero_frac=0.01)
        B = nb.random_numbers(rng, k * n, bits, spread, zero_frac=0.01)
        C0 = nb.random_numbers(rng, m * n, bits, 50)
        got = _product(api, la, True, bits, A, B, m, n, k, C0, subtract, lower)
        want = _product(api, la, False, bits, A, B, m, n, k, C0, subtract, lower)
        assert (got == want).all(), f"bits={bits} m={m} n={n} k={k} spread={spread}"


def test_static_scratch_product_allocates_nothing():
    import torch
    from limbforge_b200 import api
    torch.cuda.init()
    eng = api.Engine()
    la = api.Linalg(eng)
    rng = np.random.default_rng(11)
    bits, m, n, k = 512, 96, 80, 128
    A = nb.random_numbers(rng, k * m, bits, 40)
    B = nb.random_numbers(rng, k * n, bits, 40)
    C0 = nb.random_numbers(rng, m * n, bits, 40)
    bufs = _buffers(eng, bits, A, B, C0)
    _call(api, la, True, bits, bufs, m, n, k, True, False)          # warm: kernels loaded, tables set up
    bufs[2].upload(C0)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    _call(api, la, True, bits, bufs, m, n, k, True, False)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"device memory changed by {free0 - free1} bytes during the call"
    got = bufs[2].download()
    assert (got == _product(api, la, False, bits, A, B, m, n, k, C0, True, False)).all()


def test_static_scratch_product_takes_the_limb_kernel_when_planes_do_not_fit():
    from limbforge_b200 import api
    eng = api.Engine()
    la = api.Linalg(eng)
    bits, m, n, k = 1024, 2000, 2000, 8        # the residues alone would need far more than the static area
    rng = np.random.default_rng(7)
    A = nb.random_numbers(rng, k * m, bits, 4)
    B = nb.random_numbers(rng, k * n, bits, 4)
    C0 = nb.random_numbers(rng, m * n, bits, 4)
    got = _product(api, la, True, bits, A, B, m, n, k, C0, True, False)
    want = _product(api, la, False, bits, A, B, m, n, k, C0, True, False)
    assert (got == want).all()


def test_static_scratch_product_rejects_too_many_lines():
    from limbforge_b200 import api
    eng = api.Engine()
    la = api.Linalg(eng)
    bits, m, n, k = 128, 5000, 4000, 2
    rng = np.random.default_rng(8)
    A = nb.random_numbers(rng, k * m, bits, 4)
    B = nb.random_numbers(rng, k * n, bits, 4)
    C0 = np.zeros((m * n, bits // 32 + 3), np.uint32)
    with pytest.raises(api.InvalidArgument, match="8192 lines"):
        _product(api, la, True, bits, A, B, m, n, k, C0, False, False)
