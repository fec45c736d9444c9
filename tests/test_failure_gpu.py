"""GPU: failure detection without a GPU fault.  The tensor-core residue kernel's barrier waits are bounded: a tile
whose loads are left out (a barrier that nothing completes) gives up after a short poll limit, records error 2,
frees its tensor memory and returns, and the context stays usable for the next products, whose bits are checked.
The host-side paths of the same error word (runtime_error from the product entry points) are exercised by the
products' normal returns; nothing here traps, faults or hangs the GPU."""
import numpy as np
import pytest

from limbforge_b200 import numbers as nb

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_the_context_stays_usable(engine, oracle):
    from limbforge_b200 import api
    assert api.residue_wait_limit_test(2000) == 2
    assert api.residue_wait_limit_test(64) == 2                # twice in a row: TMEM was freed
    la = api.Linalg(engine)
    rng = np.random.default_rng(4)
    bits, m, n, k = 256, 33, 29, 70
    A = nb.random_numbers(rng, k * m, bits, 30)
    B = nb.random_numbers(rng, k * n, bits, 30)
    C = np.zeros((m * n, bits // 32 + 3), np.uint32)
    la.gemm(bits, True, A, B, m, n, k, C)
    assert la.report()["method"] == 2                          # the residue engine ran after the aborted tile
    assert (C == oracle.gemm(bits, True, A, B, m, n, k)).all()
