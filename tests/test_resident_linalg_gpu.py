"""GPU: resident exact products (Linalg::syrk / gemm recorded into a CommandBatch, linalg.hpp:190-195).

The engine, the modulus count and the line analysis are planned on the GPU inside the batch, so a
resident product must give exactly the bits of the host-array call on the same data, including data
that an earlier operation of the same batch wrote.  Covered: matrix kinds that take the residue
engine and kinds whose exponent spread sends them to the limb kernel; transposed and plain A;
lower, full and subtracting SYRK; the ticket's report; and the error rules."""
import numpy as np
import pytest

from limbforge_b200 import api
from limbforge_b200 import numbers as nb
from linalg_cases import matrix, old_entries

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def la(engine):
    return api.Linalg(engine)


def upload(engine, x, bits):
    b = engine.make_buffer(x.shape[0], bits)
    b.upload(x)
    return b


@pytest.mark.parametrize("bits,kind", [(128, "moderate"), (512, "qsc"), (256, "wide"), (64, "cancel")])
def test_resident_gemm_equals_host_call(engine, la, bits, kind):
    rng = np.random.default_rng(bits + len(kind))
    m, n, k = 37, 29, 45
    A = matrix(bits, k, m, kind, rng)                       # k x m, used transposed
    B = matrix(bits, k, n, kind, rng)
    C0 = old_entries(bits, np.zeros((m * n, bits // 32 + 3), np.uint32), rng)
    want = C0.copy()
    la.gemm(bits, True, A, B, m, n, k, want, subtract=True)
    host = la.report()
    bA, bB, bC = upload(engine, A, bits), upload(engine, B, bits), upload(engine, C0, bits)
    batch = engine.batch()
    t = la.gemm_resident(batch, True, bA, bB, m, n, k, bC, subtract=True)
    with pytest.raises(api.LogicError):
        t.report()                                          # not resolved before the batch has run
    batch.submit().wait()
    assert t.resolved()
    assert (bC.download() == want).all()
    rep = t.report()                                        # the GPU plan follows the host driver's rule
    assert (rep["method"], rep["moduli"], rep["band_bits"]) == (host["method"], host["moduli"], host["band_bits"])
    # plain (untransposed) A: rows of A are the left lines
    At = np.ascontiguousarray(A.reshape(k, m, -1).transpose(1, 0, 2).reshape(m * k, -1))
    bAt, bC2 = upload(engine, At, bits), engine.make_buffer(m * n, bits)
    batch = engine.batch()
    la.gemm_resident(batch, False, bAt, bB, m, n, k, bC2)
    batch.submit().wait()
    plain = np.zeros_like(C0)
    la.gemm(bits, True, A, B, m, n, k, plain)
    assert (bC2.download() == plain).all()


def test_plan_reads_data_written_earlier_in_the_batch(engine, la):
    """Every other row of A is scaled by 2^300 in the same batch before the product, which widens each
    line's exponent band past the residue engine's limit: the GPU plan must see the new exponents and
    choose the limb kernel."""
    bits, m, n, k = 256, 20, 24, 33
    rng = np.random.default_rng(5)
    A = matrix(bits, k, m, "moderate", rng)
    B = matrix(bits, k, n, "moderate", rng)
    scale = np.repeat(nb.power(bits, 0), k * m, axis=0)
    scale.reshape(k, m, -1)[1::2] = nb.power(bits, 300)[0]
    want = np.zeros((m * n, bits // 32 + 3), np.uint32)
    As = engine.run(bits, api.Operation.mul, A, scale)[0]
    la.gemm(bits, True, As, B, m, n, k, want)
    bA, bS, bB = upload(engine, A, bits), upload(engine, scale, bits), upload(engine, B, bits)
    bC = engine.make_buffer(m * n, bits)
    batch = engine.batch()
    batch.run(api.Operation.mul, bA, bS, None, bA)
    t = la.gemm_resident(batch, True, bA, bB, m, n, k, bC)
    batch.submit().wait()
    assert (bC.download() == want).all()
    assert t.report()["method"] == 1 and t.report()["band_bits"] == 0


@pytest.mark.parametrize("lower_only,subtract", [(True, False), (False, False), (True, True)])
def test_resident_syrk_equals_host_call(engine, la, lower_only, subtract):
    bits, rows, cols = 384, 41, 30
    rng = np.random.default_rng(11 + lower_only + 2 * subtract)
    A = matrix(bits, rows, cols, "qsc", rng)
    C0 = old_entries(bits, np.zeros((cols * cols, bits // 32 + 3), np.uint32), rng)
    want = C0.copy()
    la.syrk(bits, A, rows, cols, want, lower_only=lower_only, subtract=subtract)
    bA, bC = upload(engine, A, bits), upload(engine, C0, bits)
    batch = engine.batch()
    t = la.syrk_resident(batch, bA, rows, cols, bC, lower_only=lower_only, subtract=subtract)
    batch.submit().wait()
    assert (bC.download() == want).all()
    assert t.report()["m"] == cols


def test_resident_errors(engine, la):
    bits = 128
    b1, b2 = engine.make_buffer(16, bits), engine.make_buffer(16, bits)
    batch = engine.batch()
    with pytest.raises(api.InvalidArgument):
        la.gemm_resident(batch, False, b1, b2, 4, 4, 4, b1)            # C is A
    with pytest.raises(api.InvalidArgument):
        la.gemm_resident(batch, False, b1, b2, 8, 8, 8, engine.make_buffer(64, bits))   # undersized A
    with pytest.raises(api.InvalidArgument):
        la.syrk_resident(batch, b1, 4, 4, b2, lower_only=False, subtract=True)
    other = api.Engine()
    with pytest.raises(api.InvalidArgument):
        la.gemm_resident(other.batch(), False, b1, b2, 4, 4, 4, engine.make_buffer(16, bits))


def test_workspaces_scratch_idle_busy_and_release(engine):
    """Linalg::workspaces / release_workspaces (linalg.hpp:173-180): host-array calls leave scratch; a resident
    product's workspace is busy while its batch is unsubmitted and idle once the batch has run; release frees
    scratch and idle workspaces, returns what was retained, keeps tickets' reports and leaves later calls exact."""
    bits, m, k = 256, 24, 40
    rng = np.random.default_rng(3)
    la = api.Linalg(engine)
    A = matrix(bits, k, m, "moderate", rng)
    C1 = np.zeros((m * m, bits // 32 + 3), np.uint32)
    la.syrk(bits, A, k, m, C1, lower_only=False)
    w = la.workspaces()
    assert w["scratch_bytes"] > 0 and w["busy_workspaces"] == 0
    bA, bC = upload(engine, A, bits), upload(engine, np.zeros_like(C1), bits)
    batch = engine.batch()
    ticket = la.syrk_resident(batch, bA, k, m, bC, lower_only=False)
    w = la.workspaces()
    assert w["busy_workspaces"] == 1 and w["busy_bytes"] > 0 and w["idle_bytes"] == 0
    batch.submit().wait()
    w = la.workspaces()
    assert w["busy_workspaces"] == 0 and w["idle_bytes"] > 0
    report = ticket.report()
    orphan_batch = engine.batch()                             # recorded, then dropped unsubmitted: idle
    orphan = la.syrk_resident(orphan_batch, bA, k, m, upload(engine, np.zeros_like(C1), bits), lower_only=False)
    assert la.workspaces()["busy_workspaces"] == 1
    del orphan_batch
    before = la.workspaces()
    assert before["busy_workspaces"] == 0 and before["idle_bytes"] > w["idle_bytes"]
    assert la.release_workspaces() == before
    assert la.workspaces() == {"scratch_bytes": 0, "idle_bytes": 0, "busy_bytes": 0, "busy_workspaces": 0}
    assert ticket.report() == report
    assert (bC.download() == C1).all()
    C2 = np.zeros_like(C1)
    la.syrk(bits, A, k, m, C2, lower_only=False)
    assert (C2 == C1).all()
    del orphan


def test_product3_equals_two_products_and_reuses_its_workspace(engine):
    """BatchedLinalg::product3 (batched_linalg.hpp:99-110): C = (A B) D through an intermediate the
    BatchedLinalg keeps; bits equal two explicit resident products; the intermediate is busy until the
    batch is waited, then reused; release returns its bytes."""
    bits, count, m, n, k, q = 384, 7, 5, 4, 6, 3
    rng = np.random.default_rng(9)
    A = nb.random_complex(rng, count * m * k, bits, 20)
    B = nb.random_complex(rng, count * k * n, bits, 20)
    D = nb.random_complex(rng, count * n * q, bits, 20)
    first = api.StridedGemm(count, m, n, k, m * k, k * n, 0)
    second = api.StridedGemm(count, m, q, n, 0, n * q, m * q, negative=False)
    bl = api.BatchedLinalg(engine)

    def buf(x):
        b = engine.make_buffer(x.shape[0], bits, True)
        b.upload(x)
        return b

    bA, bB, bD = buf(A), buf(B), buf(D)
    bC = engine.make_buffer(count * m * q, bits, True)
    batch = engine.batch()
    bl.product3(batch, first, second, bA, bB, bD, bC, negative=True)
    assert bl.workspaces()["busy_workspaces"] == 1
    batch.submit().wait()
    got = bC.download()
    T = engine.make_buffer(count * m * n, bits, True)
    W = engine.make_buffer(count * m * q, bits, True)
    batch = engine.batch()
    bl.gemm_resident(batch, api.StridedGemm(count, m, n, k, m * k, k * n, m * n), bA, bB, T)
    bl.gemm_resident(batch, api.StridedGemm(count, m, q, n, m * n, n * q, m * q, negative=True), T, bD, W)
    batch.submit().wait()
    assert (got == W.download()).all()
    w = bl.workspaces()
    assert w["busy_workspaces"] == 0 and w["idle_bytes"] > 0
    batch = engine.batch()
    bl.product3(batch, first, second, bA, bB, bD, bC)
    batch.submit().wait()
    assert bl.workspaces() == w                               # the idle intermediate was reused
    assert bl.release_workspaces() == w and bl.workspaces()["idle_bytes"] == 0
    with pytest.raises(api.InvalidArgument):
        bl.product3(engine.batch(), first, api.StridedGemm(count, m, q, n + 1), bA, bB, bD, bC)
