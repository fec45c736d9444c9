"""GPU parity of the Householder QR factor, its least-squares solve and its Q applications through the C ABI
against the oracle, bit for bit (the strategy of the reference's tests/test_qr.cpp): every matrix kind at
several widths and block sizes, the special cases (zero, status and dependent columns, rank test, extreme
spreads, an entry whose scaled reflector leaves the exponent range), block boundaries, multiple right-hand
sides with a status, the augmented Levenberg-Marquardt matrix, Buffer forms, empty and invalid shapes, and
both product engines under the trailing updates."""
import numpy as np
import pytest

from limbforge_b200 import numbers as nb
from tests import qr_cases as qc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def la(engine):
    from limbforge_b200 import api
    return api.Linalg(engine)


@pytest.fixture(scope="module")
def la_limb(engine):
    from limbforge_b200 import api
    return api.Linalg(engine, api.LinalgOptions(method=1))


def opts(block, rank_bits=0, pivot=False):
    from limbforge_b200 import api
    return api.QROptions(block=block, rank_bits=rank_bits, pivot=pivot)


def bad(x, y):
    return np.nonzero((x != y).reshape(x.shape[0], -1).any(axis=1))[0][:5]


def check_factor(qr, want, label):
    assert (qr.info.rank, qr.info.reason, qr.info.status) == (want["rank"], want["reason"], want["status"]), \
        f"{label}: rank/reason/status {(qr.info.rank, qr.info.reason, qr.info.status)} want {(want['rank'], want['reason'], want['status'])}"
    if want["perm"] is not None:
        assert qr.pivoted and qr.permutation() == want["perm"], f"{label}: permutation {qr.permutation()} want {want['perm']}"
        assert qr.info.norm_recomputations == want["recomputed"], f"{label}: recomputed norms"
    for k, got in (("R", qr.r()), ("V", qr.v()), ("tau", qr.tau()), ("T", qr.t())):
        w = want[k]
        assert got.shape == w.shape and (got == w).all(), f"{label}: {k} differs at {bad(got, w)}"


def check_solves(qr, want, oracle, B, nrhs, label):
    X = qr.solve(B, nrhs)
    wx = oracle.qr_solve(want, B, nrhs)
    assert (X == wx).all(), f"{label}: solve differs at {bad(X, wx)}"
    for qt in (True, False):
        C = B.copy()
        qr.apply_q(C, nrhs, qt)
        wc = oracle.qr_apply(want, B, nrhs, qt)
        assert (C == wc).all(), f"{label}: apply {'Q^T' if qt else 'Q'} differs at {bad(C, wc)}"


SHAPES = [(1, 1, "moderate"), (3, 2, "qsc"), (33, 7, "graded"), (64, 32, "wide"), (70, 40, "spread"), (49, 33, "qsc"),
          (40, 40, "extreme"), (31, 17, "triangular"), (50, 33, "dependent")]


@pytest.mark.parametrize("bits", [64, 224, 256, 384, 512])
def test_qr_vs_oracle(la, oracle, bits):
    rng = np.random.default_rng(300 + bits)
    for i, (m, n, kind) in enumerate(SHAPES):
        A = qc.matrix(bits, m, n, kind, rng)
        for block in (32, 16, 7, 0):
            want = oracle.qr(bits, A, m, n, block)
            qr = la.factor_qr(bits, A, m, n, opts(block))
            label = f"bits={bits} {kind} {m}x{n} block {block}"
            check_factor(qr, want, label)
            nrhs = (1, 3, 5)[(i + block) % 3]
            B = qc.rhs(bits, m, nrhs, rng)
            if block == 16 and m > 3:
                B[nrhs + 1, -1] = nb.INVALID
            check_solves(qr, want, oracle, B, nrhs, label)


def test_qr_all_widths(la, oracle):
    rng = np.random.default_rng(5)
    for bits in range(64, 1025, 32):
        A = qc.matrix(bits, 21, 9, "qsc", rng)
        want = oracle.qr(bits, A, 21, 9, 4)
        qr = la.factor_qr(bits, A, 21, 9, opts(4))
        check_factor(qr, want, f"bits={bits}")
        B = qc.rhs(bits, 21, 2, rng)
        check_solves(qr, want, oracle, B, 2, f"bits={bits}")


def test_qr_special_cases(la, oracle):
    bits = 256
    rng = np.random.default_rng(77)
    for label, A, m, n, rank_bits, expect in qc.special_cases(bits, rng):
        for block in (16, 7, 1):
            want = oracle.qr(bits, A, m, n, block, rank_bits)
            qr = la.factor_qr(bits, A, m, n, opts(block, rank_bits))
            check_factor(qr, want, f"{label} block {block}")
            if expect is not None:
                assert qr.info.rank == expect, label
            assert qr.full_rank() == (want["rank"] == n)
            B = qc.rhs(bits, m, 3, rng)
            check_solves(qr, want, oracle, B, 3, f"{label} block {block}")


def test_qr_block_boundaries(la, oracle):
    rng = np.random.default_rng(17)
    bits = 224
    for n in (15, 16, 17, 31, 32, 33, 63, 64, 65):
        m = n + n // 2 + 1
        A = qc.matrix(bits, m, n, "qsc" if n % 2 else "moderate", rng)
        for block in (16, 32):
            want = oracle.qr(bits, A, m, n, block)
            check_factor(la.factor_qr(bits, A, m, n, opts(block)), want, f"{m}x{n} block {block}")


def test_qr_limb_kernel_updates(la_limb, oracle):
    """The trailing updates on the generic limb kernel give the same factor."""
    rng = np.random.default_rng(23)
    for bits in (128, 256):
        A = qc.matrix(bits, 90, 48, "qsc", rng)
        want = oracle.qr(bits, A, 90, 48, 16)
        qr = la_limb.factor_qr(bits, A, 90, 48, opts(16))
        check_factor(qr, want, f"limb kernel bits={bits}")
        check_solves(qr, want, oracle, qc.rhs(bits, 90, 2, rng), 2, "limb kernel")


def test_qr_qsc_least_squares(la, oracle):
    """QSC-like J (m = 2n) at 256 bits, the shape of the reference's QR benchmark, scaled to the oracle's budget."""
    rng = np.random.default_rng(800)
    bits, m, n = 256, 400, 200
    A = qc.matrix(bits, m, n, "qsc", rng)
    want = oracle.qr(bits, A, m, n, 32)
    qr = la.factor_qr(bits, A, m, n, opts(32))
    check_factor(qr, want, "QSC 400x200")
    assert qr.info.blocks == 7 and qr.info.gpu_updates >= 6
    check_solves(qr, want, oracle, qc.rhs(bits, m, 4, rng), 4, "QSC 400x200")


def test_qr_augmented(la, oracle):
    bits, m, n = 256, 37, 21
    rng = np.random.default_rng(37)
    J = qc.matrix(bits, m, n, "qsc", rng)
    d = nb.random_numbers(rng, n, bits, 6)
    d[:, bits // 32 + 1] = 1
    S = qc.augmented(bits, J, m, n, d)
    want = oracle.qr(bits, S, m + n, n, 8)
    a = la.factor_qr_augmented(bits, J, m, n, d, opts(8))
    check_factor(a, want, "augmented")
    check_factor(la.factor_qr(bits, S, m + n, n, opts(8)), want, "stacked")
    B = qc.rhs(bits, m + n, 2, rng)
    check_solves(a, want, oracle, B, 2, "augmented")


def test_qr_buffers(engine, la, oracle):
    bits, m, n, nrhs = 256, 45, 20, 3
    rng = np.random.default_rng(45)
    A = qc.matrix(bits, m, n, "moderate", rng)
    B = qc.rhs(bits, m, nrhs, rng)
    want = oracle.qr(bits, A, m, n, 8)
    bA = engine.make_buffer(m * n, bits)
    bA.upload(A)
    qr = la.factor_qr_buffer(bA, m, n, opts(8))
    check_factor(qr, want, "buffer factor")
    bB, bX = engine.make_buffer(m * nrhs, bits), engine.make_buffer(n * nrhs, bits)
    bB.upload(B)
    qr.solve_buffers(bB, nrhs, bX)
    assert (bX.download() == oracle.qr_solve(want, B, nrhs)).all()
    qr.apply_q_buffer(bB, nrhs, True)
    assert (bB.download() == oracle.qr_apply(want, B, nrhs, True)).all()


def test_qr_empty_and_invalid(la):
    from limbforge_b200 import api
    bits = 256
    w = bits // 32 + 3
    e = la.factor_qr(bits, np.zeros((0, w), np.uint32), 0, 0)
    assert e.full_rank() and e.info.rank == 0
    e.solve(np.zeros((0, w), np.uint32), 3)
    z = la.factor_qr(bits, np.zeros((5 * 0, w), np.uint32), 5, 0)
    assert z.info.rank == 0 and z.full_rank()
    A = np.zeros((12, w), np.uint32)
    with pytest.raises(api.InvalidArgument):
        la.factor_qr(bits, A, 3, 4)
    with pytest.raises(api.InvalidArgument):
        la.factor_qr(bits, A, 4, 3, opts(8, rank_bits=-1))
    with pytest.raises(api.InvalidArgument):
        la.factor_qr(100, A, 4, 3)


@pytest.mark.parametrize("bits", [64, 256, 384])
def test_qr_pivoted_vs_oracle(la, oracle, bits):
    rng = np.random.default_rng(400 + bits)
    for i, (m, n, kind) in enumerate([(1, 1, "moderate"), (5, 3, "qsc"), (33, 7, "graded"), (60, 30, "qsc"), (64, 32, "wide"),
                                      (70, 40, "spread"), (150, 60, "moderate")]):
        A = qc.matrix(bits, m, n, kind, rng)
        for block in (16, 7, 0):
            want = oracle.qr(bits, A, m, n, block, 0, pivot=True)
            qr = la.factor_qr(bits, A, m, n, opts(block, pivot=True))
            label = f"pivoted bits={bits} {kind} {m}x{n} block {block}"
            check_factor(qr, want, label)
            nrhs = (1, 3, 5)[(i + block) % 3]
            check_solves(qr, want, oracle, qc.rhs(bits, m, nrhs, rng), nrhs, label)


def test_qr_pivoted_fixtures(la, oracle):
    bits = 256
    N = bits // 32
    rng = np.random.default_rng(8)
    cases = [("dependent", qc.matrix(bits, 41, 7, "dependent", rng), 41, 7, bits // 2, 5),
             ("dependent 90x40", qc.matrix(bits, 90, 40, "dependent", rng), 90, 40, bits // 2, 38)]
    A = qc.matrix(bits, 30, 12, "moderate", rng)
    A[2::12] = 0
    A[7::12] = 0
    cases.append(("zero columns 2, 7", A, 30, 12, 0, 10))
    A = qc.matrix(bits, 25, 9, "moderate", rng)
    for r in range(25):
        A[r * 9 + 6] = A[r * 9 + 2]
        A[r * 9 + 8] = A[r * 9 + 2]
    cases.append(("duplicate columns", A, 25, 9, bits // 2, 7))
    A = qc.matrix(bits, 25, 10, "moderate", rng)
    A[7 * 10 + 4, N + 2] = nb.INVALID
    cases.append(("status at (7,4)", A, 25, 10, 0, 0))
    A = qc.matrix(bits, 80, 20, "moderate", rng)
    for j in (5, 13):
        t = nb.random_numbers(rng, 80, bits, 4)
        t[:, N] = (nb.exponent(t) - (bits // 4 + 10)).astype(np.int32).view(np.uint32)
        A[j::20] = oracle.elementwise(bits, 0, np.ascontiguousarray(A[j - 1::20]), t)
    cases.append(("nearly parallel columns", A, 80, 20, 0, None))
    cases.append(("QSC-like", qc.matrix(bits, 300, 150, "qsc", rng), 300, 150, 0, None))
    for label, A, m, n, rank_bits, expect in cases:
        for block in (16, 7):
            want = oracle.qr(bits, A, m, n, block, rank_bits, pivot=True)
            qr = la.factor_qr(bits, A, m, n, opts(block, rank_bits, pivot=True))
            check_factor(qr, want, f"{label} block {block}")
            if expect is not None:
                assert qr.info.rank == expect, label
            if label == "nearly parallel columns":
                assert qr.info.norm_recomputations > 0
            check_solves(qr, want, oracle, qc.rhs(bits, m, 3, rng), 3, f"{label} block {block}")


# ---- complex QR (linalg_complex.mm): the factor, least squares and Q / Q^H against the oracle's complex sequence
def check_cfactor(qr, want, label):
    assert qr.complex
    assert (qr.info.rank, qr.info.reason, qr.info.status) == (want["rank"], want["reason"], want["status"]), label
    for k, got in (("R", qr.r()), ("V", qr.v()), ("tau", qr.tau()), ("T", qr.t())):
        w = want[k]
        assert got.shape == w.shape and (got == w).all(), f"{label}: {k} differs at {bad(got.reshape(got.shape[0], -1), w.reshape(w.shape[0], -1))}"


def check_csolves(qr, want, oracle, B, nrhs, label):
    X = qr.solve(B, nrhs)
    assert (X == oracle.qr_complex_solve(want, B, nrhs)).all(), f"{label}: solve"
    for adj in (True, False):
        C = B.copy()
        qr.apply_q(C, nrhs, adj)
        assert (C == oracle.qr_complex_apply(want, B, nrhs, adj)).all(), f"{label}: apply {'Q^H' if adj else 'Q'}"


@pytest.mark.parametrize("bits", [64, 256, 416])
def test_qr_complex_vs_oracle(la, oracle, bits):
    rng = np.random.default_rng(600 + bits)
    for i, (m, n, kind) in enumerate([(1, 1, "moderate"), (3, 2, "qsc"), (33, 7, "graded"), (40, 21, "wide"), (50, 24, "spread"),
                                      (30, 17, "triangular"), (41, 7, "dependent")]):
        A = qc.complex_matrix(bits, m, n, kind, rng)
        for block in (16, 5, 0):
            want = oracle.qr_complex(bits, A, m, n, block)
            qr = la.factor_qr_complex(bits, A, m, n, opts(block))
            label = f"complex bits={bits} {kind} {m}x{n} block {block}"
            check_cfactor(qr, want, label)
            nrhs = (1, 2, 3)[(i + block) % 3]
            B = qc.complex_rhs(bits, m, nrhs, rng)
            if block == 5 and m > 3:
                B[nrhs + 1, 1, -1] = nb.INVALID
            check_csolves(qr, want, oracle, B, nrhs, label)


def test_qr_complex_special_cases(la, oracle):
    bits = 256
    N = bits // 32
    rng = np.random.default_rng(61)
    cases = []
    A = qc.complex_matrix(bits, 20, 9, "moderate", rng)
    A[3::9] = 0
    cases.append(("zero column 3", A, 20, 9, 0))
    A = qc.complex_matrix(bits, 25, 10, "moderate", rng)
    A[7 * 10 + 4, 1, N + 2] = nb.INVALID
    cases.append(("status at (7,4)", A, 25, 10, 0))
    cases.append(("dependent, rank_bits", qc.complex_matrix(bits, 41, 7, "dependent", rng), 41, 7, bits // 2))
    A = qc.complex_matrix(bits, 6, 3, "moderate", rng)
    A[0::3] = 0
    A[0, 1] = nb.power(bits, 3)[0]
    cases.append(("imaginary diagonal, zero below", A, 6, 3, 0))
    w = bits // 32 + 3
    R = qc.matrix(bits, 30, 12, "qsc", rng)
    A = np.zeros((30 * 12, 2, w), np.uint32)
    A[:, 0] = R
    cases.append(("real input", A, 30, 12, 0))
    for label, A, m, n, rank_bits in cases:
        for block in (4, 16):
            want = oracle.qr_complex(bits, A, m, n, block, rank_bits)
            qr = la.factor_qr_complex(bits, A, m, n, opts(block, rank_bits))
            check_cfactor(qr, want, f"{label} block {block}")
            check_csolves(qr, want, oracle, qc.complex_rhs(bits, m, 2, rng), 2, f"{label} block {block}")
    # the real input gives the real factor in the real parts
    real = la.factor_qr(bits, R, 30, 12, opts(4))
    cq = la.factor_qr_complex(bits, cases[-1][1], 30, 12, opts(4))
    assert (cq.r()[:, 0] == real.r()).all() and (cq.r()[:, 1] == 0).all()


def check_cpivot(qr, want, label):
    assert qr.pivoted and qr.permutation() == want["perm"], f"{label}: permutation {qr.permutation()} want {want['perm']}"
    assert qr.info.norm_recomputations == want["recomputed"], f"{label}: recomputed norms"
    check_cfactor(qr, want, label)


@pytest.mark.parametrize("bits", [64, 256, 416])
def test_qr_complex_pivoted_vs_oracle(la, oracle, bits):
    rng = np.random.default_rng(700 + bits)
    for i, (m, n, kind) in enumerate([(1, 1, "moderate"), (5, 3, "qsc"), (33, 7, "graded"), (40, 21, "wide"), (50, 24, "spread"),
                                      (41, 7, "dependent"), (90, 40, "qsc")]):
        A = qc.complex_matrix(bits, m, n, kind, rng)
        for block in (16, 5, 0):
            want = oracle.qr_complex(bits, A, m, n, block, 0, pivot=True)
            qr = la.factor_qr_complex(bits, A, m, n, opts(block, pivot=True))
            label = f"pivoted complex bits={bits} {kind} {m}x{n} block {block}"
            check_cpivot(qr, want, label)
            nrhs = (1, 2, 3)[(i + block) % 3]
            check_csolves(qr, want, oracle, qc.complex_rhs(bits, m, nrhs, rng), nrhs, label)


def test_qr_complex_pivoted_fixtures(la, oracle):
    bits = 256
    N = bits // 32
    rng = np.random.default_rng(71)
    cases = [("dependent, rank_bits", qc.complex_matrix(bits, 41, 7, "dependent", rng), 41, 7, bits // 2)]
    A = qc.complex_matrix(bits, 30, 12, "moderate", rng)
    A[2::12] = 0
    A[7::12] = 0
    cases.append(("zero columns 2, 7", A, 30, 12, 0))
    A = qc.complex_matrix(bits, 25, 9, "moderate", rng)
    for r in range(25):
        A[r * 9 + 6] = A[r * 9 + 2]
    cases.append(("duplicate columns", A, 25, 9, bits // 2))
    A = qc.complex_matrix(bits, 25, 10, "moderate", rng)
    A[7 * 10 + 4, 1, N + 2] = nb.INVALID
    cases.append(("status at (7,4)", A, 25, 10, 0))
    A = qc.complex_matrix(bits, 80, 20, "moderate", rng)
    for j in (5, 13):                                          # nearly parallel columns: collapsed norms are recomputed
        t = nb.random_complex(rng, 80, bits, 4)
        for part in (0, 1):
            t[:, part, N] = (nb.exponent(t[:, part]) - (bits // 4 + 10)).astype(np.int32).view(np.uint32)
        A[j::20] = oracle.elementwise(bits, 4, np.ascontiguousarray(A[j - 1::20]), t)
    cases.append(("nearly parallel columns", A, 80, 20, 0))
    w = bits // 32 + 3
    R = qc.matrix(bits, 30, 12, "qsc", rng)
    A = np.zeros((30 * 12, 2, w), np.uint32)
    A[:, 0] = R
    cases.append(("real input", A, 30, 12, 0))
    for label, A, m, n, rank_bits in cases:
        for block in (4, 16):
            want = oracle.qr_complex(bits, A, m, n, block, rank_bits, pivot=True)
            qr = la.factor_qr_complex(bits, A, m, n, opts(block, rank_bits, pivot=True))
            check_cpivot(qr, want, f"{label} block {block}")
            if label == "nearly parallel columns":
                assert qr.info.norm_recomputations > 0
            check_csolves(qr, want, oracle, qc.complex_rhs(bits, m, 2, rng), 2, f"{label} block {block}")
    # the real input gives the real pivoted factor in the real parts
    real = la.factor_qr(bits, R, 30, 12, opts(4, pivot=True))
    cq = la.factor_qr_complex(bits, cases[-1][1], 30, 12, opts(4, pivot=True))
    assert cq.permutation() == real.permutation()
    assert (cq.r()[:, 0] == real.r()).all() and (cq.r()[:, 1] == 0).all()


def test_qr_large_factor_parity(la, oracle):
    """Whole factors and solutions at bench-like sizes: real 1000 x 500 and complex 400 x 200, QSC-like, block 32."""
    bits = 256
    rng = np.random.default_rng(901)
    A = qc.matrix(bits, 1000, 500, "qsc", rng)
    want = oracle.qr(bits, A, 1000, 500, 32)
    qr = la.factor_qr(bits, A, 1000, 500, opts(32))
    check_factor(qr, want, "real 1000x500")
    check_solves(qr, want, oracle, qc.rhs(bits, 1000, 4, rng), 4, "real 1000x500")
    Z = qc.complex_matrix(bits, 400, 200, "qsc", rng)
    wantc = oracle.qr_complex(bits, Z, 400, 200, 32)
    cq = la.factor_qr_complex(bits, Z, 400, 200, opts(32))
    check_cfactor(cq, wantc, "complex 400x200")
    check_csolves(cq, wantc, oracle, qc.complex_rhs(bits, 400, 4, rng), 4, "complex 400x200")
