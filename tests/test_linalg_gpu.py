"""GPU parity of the exact dense products and factorizations through the C ABI against the
C oracle, bit for bit (tests/test_linalg.cpp and tests/test_cholesky.cpp strategies): matrix
kinds with several exponent bands, cancellation, sparsity, statuses, ties and saturation; updates
with adversarial old entries; degenerate shapes; blocked Cholesky with every block size and its
failure cases; multi-RHS triangular solves; both product engines give identical bits."""
import numpy as np
import pytest

from limbforge_b200 import numbers as nb
from linalg_cases import KINDS, matrix, old_entries, rhs, spd

pytestmark = pytest.mark.gpu


def same(x, y):
    return x.shape == y.shape and bool((x == y).all())


def bad(x, y):
    return np.nonzero((x != y).reshape(x.shape[0], -1).any(axis=1))[0][:5]


@pytest.fixture(scope="module")
def la(engine):
    from limbforge_b200 import api
    return api.Linalg(engine)


@pytest.fixture(scope="module")
def la_limb(engine):
    from limbforge_b200 import api
    return api.Linalg(engine, api.LinalgOptions(method=1))


def transpose(A, rows, cols):
    return np.ascontiguousarray(A.reshape(rows, cols, -1).transpose(1, 0, 2).reshape(rows * cols, -1))


@pytest.mark.parametrize("bits", [64, 256, 512])
@pytest.mark.parametrize("kind", KINDS)
def test_products_vs_oracle(la, oracle, bits, kind):
    rng = np.random.default_rng(1000 + bits + KINDS.index(kind))
    for s in (7, 33):
        rows = 2 * s + 1 if kind in ("qsc", "cancel") else s
        A = matrix(bits, rows, s, kind, rng)
        for lower in (True, False):
            sentinel = np.zeros((s * s, bits // 32 + 3), np.uint32)
            sentinel[:] = nb.power(bits, 12345)[0]
            sentinel[:, -1] = nb.INVALID
            C = sentinel.copy()
            la.syrk(bits, A, rows, s, C, lower_only=lower)
            want = oracle.syrk(bits, A, rows, s, C=sentinel, lower_only=lower)   # upper left as the sentinel
            assert same(C, want), f"syrk {kind} s={s} lower={lower} bad {bad(C, want)}"
        m, n, k = s, s + 3, rows
        L = matrix(bits, k, m, kind, rng)
        R = matrix(bits, k, n, kind, rng)
        C = np.zeros((m * n, bits // 32 + 3), np.uint32)
        la.gemm(bits, True, L, R, m, n, k, C)
        want = oracle.gemm(bits, True, L, R, m, n, k)
        assert same(C, want), f"gemm AT {kind} s={s} bad {bad(C, want)}"
        C2 = np.zeros_like(C)
        la.gemm(bits, False, transpose(L, k, m), R, m, n, k, C2)
        assert same(C2, want), f"gemm A {kind} s={s}"
        old = old_entries(bits, want, rng)
        Cu = old.copy()
        la.gemm(bits, True, L, R, m, n, k, Cu, subtract=True)
        wu = oracle.gemm(bits, True, L, R, m, n, k, C=old, subtract=True)
        assert same(Cu, wu), f"gemm update {kind} s={s} bad {bad(Cu, wu)}"
        P = oracle.syrk(bits, A, rows, s, lower_only=False)
        old = old_entries(bits, P, rng)
        Cs = old.copy()
        la.syrk(bits, A, rows, s, Cs, lower_only=True, subtract=True)
        ws = oracle.syrk(bits, A, rows, s, C=old, lower_only=True, subtract=True)
        assert same(Cs, ws), f"syrk update {kind} s={s} bad {bad(Cs, ws)}"


@pytest.mark.parametrize("bits", [64, 256, 512, 1024])
@pytest.mark.parametrize("kind", KINDS)
def test_limb_kernel_products_vs_oracle(la_limb, oracle, bits, kind):
    """The tiled limb kernel (per-output exact windows, cluster method for wide outputs) on every matrix kind:
    GEMM updates with adversarial old entries, plain GEMM and SYRK, against the oracle."""
    rng = np.random.default_rng(7000 + bits + KINDS.index(kind))
    for m, n, k in ((9, 13, 21), (17, 8, 40)):
        L = matrix(bits, k, m, kind, rng)
        R = matrix(bits, k, n, kind, rng)
        want = oracle.gemm(bits, True, L, R, m, n, k)
        C = np.zeros((m * n, bits // 32 + 3), np.uint32)
        la_limb.gemm(bits, True, L, R, m, n, k, C)
        assert same(C, want), f"gemm {kind} bad {bad(C, want)}"
        old = old_entries(bits, want, rng)
        Cu = old.copy()
        la_limb.gemm(bits, True, L, R, m, n, k, Cu, subtract=True)
        wu = oracle.gemm(bits, True, L, R, m, n, k, C=old, subtract=True)
        assert same(Cu, wu), f"gemm update {kind} bad {bad(Cu, wu)}"
        S = np.zeros((m * m, bits // 32 + 3), np.uint32)
        la_limb.syrk(bits, L, k, m, S, lower_only=True)
        assert same(S, oracle.syrk(bits, L, k, m, C=np.zeros_like(S), lower_only=True)), f"syrk {kind}"
    assert la_limb.report()["method"] == 1


def test_limb_and_auto_engines_agree(la, la_limb, oracle):
    bits, m, n, k = 512, 40, 37, 129
    rng = np.random.default_rng(3)
    L = nb.random_numbers(rng, k * m, bits, 40, zero_frac=0.005)
    R = nb.random_numbers(rng, k * n, bits, 40, zero_frac=0.005)
    C0 = nb.random_numbers(rng, m * n, bits, 60)
    a, b = C0.copy(), C0.copy()
    la.gemm(bits, True, L, R, m, n, k, a, subtract=True)
    la_limb.gemm(bits, True, L, R, m, n, k, b, subtract=True)
    assert la_limb.report()["method"] == 1
    assert same(a, b)
    assert same(a, oracle.gemm(bits, True, L, R, m, n, k, C=C0, subtract=True))


def test_degenerate_shapes(la):
    from limbforge_b200.api import InvalidArgument
    bits = 256
    C = np.zeros((9, 11), np.uint32)
    C[:] = nb.power(bits, 3)[0]
    la.syrk(bits, np.zeros((0, 11), np.uint32), 0, 3, C, lower_only=False)
    assert (C == 0).all()                                  # K = 0: canonical zeros
    la.gemm(bits, False, np.zeros((1, 11), np.uint32), np.zeros((1, 11), np.uint32), 0, 0, 5, np.zeros((1, 11), np.uint32))
    C = np.zeros((4, 11), np.uint32)
    C[:] = nb.power(bits, 7)[0]
    keep = C.copy()
    la.gemm(bits, False, np.zeros((1, 11), np.uint32), np.zeros((1, 11), np.uint32), 2, 2, 0, C, subtract=True)
    assert same(C, keep)                                   # empty K: an update leaves C unchanged
    with pytest.raises(InvalidArgument):
        la.syrk(bits, np.zeros((4, 11), np.uint32), 2, 2, C, lower_only=False, subtract=True)
    with pytest.raises(InvalidArgument):
        la.gemm(100, False, C, C, 1, 1, 1, C)


def test_saturated_sums_and_tight_bounds(la, oracle):
    """Saturated sums over growing K (test_linalg.cpp:175-177) stress the accumulator widths."""
    bits = 128
    rng = np.random.default_rng(5)
    K = 1
    while K <= 600:
        A = matrix(bits, K, 5, "saturated", rng)
        C = np.zeros((25, bits // 32 + 3), np.uint32)
        la.syrk(bits, A, K, 5, C, lower_only=False)
        assert same(C, oracle.syrk(bits, A, K, 5, lower_only=False)), f"K={K}"
        K = K * 2 + (K % 3 == 1)


def test_gemm_update_512bit_1024_sampled(la, oracle):
    """512-bit A^T B update on a 1024 x 1024 x 1024 problem with exponents in [-40, 40] and 0.5% zeros:
    every output computed on the GPU, 16 full rows checked against the oracle, and the
    SYRK lower triangle sampled too."""
    bits, n = 512, 1024
    rng = np.random.default_rng(2)
    A = nb.random_numbers(rng, n * n, bits, 40, zero_frac=0.005)
    B = nb.random_numbers(rng, n * n, bits, 40, zero_frac=0.005)
    C0 = nb.random_numbers(rng, n * n, bits, 40)
    C = C0.copy()
    la.gemm(bits, True, A, B, n, n, n, C, subtract=True)
    rows = rng.choice(n, 16, replace=False)
    for r in rows:
        want = oracle.gemm(bits, True, A, B, n, n, n, C=C0, subtract=True, rows=(int(r), int(r) + 1))
        assert same(C[r * n:(r + 1) * n], want[r * n:(r + 1) * n]), f"row {r}"
    S = np.zeros_like(C0)
    la.syrk(bits, A, n, n, S, lower_only=True)
    for r in rows[:6]:
        want = oracle.syrk(bits, A, n, n, lower_only=True, lines=(int(r), int(r) + 1))
        assert same(S[r * n:r * n + r + 1], want[r * n:r * n + r + 1]), f"syrk row {r}"


# ---------------------------------------------------------------- factorizations
RUNS = [("default", 32), ("block 16", 16), ("block 7", 7), ("block 1", 1), ("single block", 0)]


@pytest.mark.parametrize("bits", [128, 256])
@pytest.mark.parametrize("kind,n", [("moderate", 1), ("qsc", 2), ("graded", 7), ("qsc", 33), ("wide", 40),
                                    ("banded", 50), ("rank_deficient", 12), ("moderate", 70)])
def test_cholesky_and_solves_vs_oracle(la, oracle, bits, kind, n):
    from limbforge_b200.api import FactorOptions
    rng = np.random.default_rng(bits * 7 + n)
    A = spd(oracle, bits, n, kind, rng)
    for name, blk in RUNS:
        if blk == 1 and n > 40:
            continue
        L = np.zeros_like(A)
        info = la.cholesky(bits, A, n, L, FactorOptions(block=blk))
        WL, winfo = oracle.cholesky(bits, A, n, blk)
        assert (info.pivot, info.pivot_sign, info.pivot_status) == winfo, f"{kind} n={n} {name}"
        assert same(L, WL), f"cholesky {kind} n={n} {name} bad {bad(L, WL)}"
        if winfo[0] < n:
            continue
        nrhs = 3
        B = rhs(bits, n, nrhs, rng)
        for passes in (3, 1, 2):
            X = np.zeros_like(B)
            if passes == 3:
                la.cholesky_solve(bits, L, n, B, nrhs, X, FactorOptions(block=blk))
            else:
                la.trsm(bits, passes == 2, L, n, B, nrhs, X, FactorOptions(block=blk))
            W = oracle.solve(bits, L, n, B, nrhs, blk, passes)
            assert same(X, W), f"solve passes={passes} {kind} n={n} {name} bad {bad(X, W)}"


@pytest.mark.parametrize("bits,kind,n", [(64, "qsc", 35), (416, "moderate", 40), (416, "graded", 33), (1024, "qsc", 36),
                                         (1024, "wide", 12)])
def test_cholesky_and_solves_wide_limbs(la, oracle, bits, kind, n):
    """Panels and solves at widths whose exact-dot windows span one, two and three columns per lane."""
    from limbforge_b200.api import FactorOptions
    rng = np.random.default_rng(bits + n)
    A = spd(oracle, bits, n, kind, rng)
    L = np.zeros_like(A)
    info = la.cholesky(bits, A, n, L, FactorOptions(block=32))
    WL, winfo = oracle.cholesky(bits, A, n, 32)
    assert (info.pivot, info.pivot_sign, info.pivot_status) == winfo
    assert same(L, WL), f"cholesky bad {bad(L, WL)}"
    if winfo[0] < n:
        return
    B = rhs(bits, n, 4, rng)
    X = np.zeros_like(B)
    la.cholesky_solve(bits, L, n, B, 4, X, FactorOptions(block=32))
    assert same(X, oracle.solve(bits, L, n, B, 4, 32, 3))


def test_cholesky_failures(la, oracle):
    from limbforge_b200.api import FactorOptions
    bits = 192
    one, two = nb.power(bits, 0)[0], nb.power(bits, 1)[0]
    cases = [(np.stack([one, one, one, one]), 2), (np.stack([one, two, two, one]), 2), (nb.negate(one[None]), 1),
             (np.zeros((9, bits // 32 + 3), np.uint32), 3)]
    rng = np.random.default_rng(9)
    A = spd(oracle, bits, 40, "moderate", rng)
    A[37 * 40 + 37] = nb.power(bits, 40, -1)[0]
    cases.append((A, 40))
    A = spd(oracle, bits, 40, "moderate", rng)
    A[20 * 40 + 5, -1] = nb.INVALID
    cases.append((A, 40))
    A = spd(oracle, bits, 40, "qsc", rng)
    A[0, -1] = nb.EXPONENT_OVERFLOW
    cases.append((A, 40))
    A = spd(oracle, bits, 40, "moderate", rng)
    for j in range(40):
        A[max(j, 23) * 40 + min(j, 23)] = 0
    cases.append((A, 40))
    for A, n in cases:
        A = np.ascontiguousarray(A)
        for blk in (32, 4):
            L = np.zeros_like(A)
            info = la.cholesky(bits, A, n, L, FactorOptions(block=blk))
            WL, winfo = oracle.cholesky(bits, A, n, blk)
            assert (info.pivot, info.pivot_sign, info.pivot_status) == winfo
            assert same(L, WL), f"n={n} block={blk} bad {bad(L, WL)}"
    # trsm with a zero diagonal entry: division_by_zero propagates
    n, nrhs = 20, 2
    Lz = np.zeros((n * n, bits // 32 + 3), np.uint32)
    for i in range(n):
        Lz[i * n:i * n + i + 1] = nb.random_numbers(rng, i + 1, bits, 3)
    Lz[9 * n + 9] = 0
    B = rhs(bits, n, nrhs, rng)
    for t in (False, True):
        X = np.zeros_like(B)
        la.trsm(bits, t, Lz, n, B, nrhs, X, FactorOptions(block=4))
        assert same(X, oracle.solve(bits, Lz, n, B, nrhs, 4, 2 if t else 1))


def test_cholesky_in_place_and_empty(la, oracle):
    from limbforge_b200.api import FactorOptions
    bits, n = 256, 24
    rng = np.random.default_rng(11)
    A = spd(oracle, bits, n, "moderate", rng)
    WL, _ = oracle.cholesky(bits, A, n, 8)
    M = A.copy()
    la.cholesky(bits, M, n, M, FactorOptions(block=8))       # L may equal A
    assert same(M, WL)
    info = la.cholesky(bits, np.zeros((1, 11), np.uint32), 0, np.zeros((1, 11), np.uint32))
    assert info.pivot == 0


def uniform_pm1(rng, bits, count):
    """Entries uniform in [-1, 1] at full precision: random sign and significand, exponent -g with g geometric."""
    x = nb.random_numbers(rng, count, bits, 0)
    x[:, bits // 32] = (-rng.geometric(0.5, size=count)).astype(np.int32).view(np.uint32)
    return x


def test_cholesky_512_blocked_full_factor(engine, la, oracle):
    """The benchmark's construction at n = 512 (A = RN(G^T G) + n I, G uniform in [-1, 1], 256 bits, block 32):
    every entry of the factor and of an 8-RHS solve against the oracle.  Fifteen trailing updates of the
    residue engine (K = 32) run between the panels."""
    from limbforge_b200.api import FactorOptions, Operation
    bits, n, nrhs = 256, 512, 8
    rng = np.random.default_rng(2048)
    G = uniform_pm1(rng, bits, n * n)
    A = np.zeros_like(G)
    la.syrk(bits, G, n, n, A, lower_only=False)
    W = oracle.syrk(bits, G, n, n, lower_only=False, lines=(0, 3))
    for i in range(3):                                        # rows 0..2 up to the diagonal, as the oracle's lines
        assert same(A[i * n:i * n + i + 1], W[i * n:i * n + i + 1])
    diag = np.ascontiguousarray(A[np.arange(n) * (n + 1)])
    A[np.arange(n) * (n + 1)] = engine.run(bits, Operation.add, diag, nb.power(bits, 9, count=n))[0]
    L = np.zeros_like(A)
    info = la.cholesky(bits, A, n, L, FactorOptions(block=32))
    WL, winfo = oracle.cholesky(bits, A, n, 32)
    assert (info.pivot, info.pivot_sign, info.pivot_status) == winfo == (n, 0, 0)
    assert same(L, WL), f"factor rows {bad(L, WL)}"
    B = uniform_pm1(rng, bits, n * nrhs)
    X = np.zeros_like(B)
    la.cholesky_solve(bits, L, n, B, nrhs, X, FactorOptions(block=32))
    assert same(X, oracle.solve(bits, L, n, B, nrhs, 32, 3))
