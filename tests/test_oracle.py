"""CPU: pin the C oracle (oracle/lf_oracle.c) before trusting it.

* against the golden vectors (tests/golden/arith_golden.npz: the reference tests' fixture
  classes, outputs from the reference's own core.hpp / exact_dot_add, MPFR-checked);
* against the reference's CPU arithmetic compiled from its sources (oracle/_ref) on random
  inputs at all 31 widths, when that build is present;
* against independent MPFR replays of the Cholesky / triangular-solve / batched-LU /
  strided-GEMM sequences (the reference's test_cholesky.cpp, test_batched4.cpp and
  section9_cases.hpp replays) on small cases;
* and a planted mistake in an oracle output must be caught by the comparison.
"""
import numpy as np
import pytest

from limbforge_b200 import numbers as nb
from oracle.oracle import Mpfr, Reference

GOLDEN_WIDTHS = [64, 96, 128, 224, 256, 384, 512, 1024]


def same(x, y):
    return x.shape == y.shape and bool((x == y).all())


@pytest.mark.parametrize("bits", GOLDEN_WIDTHS)
def test_oracle_matches_golden_real(oracle, golden, bits):
    a, b, roots = golden[f"real_{bits}_a"], golden[f"real_{bits}_b"], golden[f"real_{bits}_roots"]
    for op in (0, 1, 2, 3, 7, 8):
        x = roots if op == 8 else a
        got = oracle.elementwise(bits, op, x, b)
        want = golden[f"real_{bits}_{op}_out"]
        bad = np.nonzero((got != want).any(axis=1))[0]
        assert not len(bad), f"bits={bits} op={op} first bad case {bad[:5]}"


@pytest.mark.parametrize("bits", GOLDEN_WIDTHS)
def test_oracle_matches_golden_fused_and_complex(oracle, golden, bits):
    fa, fb, fc = golden[f"fused_{bits}_a"], golden[f"fused_{bits}_b"], golden[f"fused_{bits}_c"]
    for op in (9, 10):
        assert same(oracle.elementwise(bits, op, fa, fb, fc), golden[f"fused_{bits}_{op}_out"]), f"fma op {op}"
    ca, cb, cc = golden[f"cx_{bits}_a"], golden[f"cx_{bits}_b"], golden[f"cx_{bits}_c"]
    for op in (4, 5, 6, 11, 12):
        assert same(oracle.elementwise(bits, op, ca, cb, cc), golden[f"cx_{bits}_{op}_out"]), f"complex op {op}"


@pytest.mark.parametrize("bits", GOLDEN_WIDTHS)
def test_oracle_matches_golden_dots(oracle, golden, bits):
    q = 0
    while f"dot_{bits}_{q}_a" in golden:
        a, b, c = golden[f"dot_{bits}_{q}_a"], golden[f"dot_{bits}_{q}_b"], golden[f"dot_{bits}_{q}_c"]
        has_c, sub = (int(v) for v in golden[f"dot_{bits}_{q}_meta"])
        got = oracle.exact_dot_add(bits, c if has_c else None, sub, a, 1, b, 1, a.shape[0])
        assert same(got, golden[f"dot_{bits}_{q}_out"]), f"dot case {q}"
        q += 1
    assert q > 50


def test_planted_mistake_is_caught(oracle, golden):
    """Fault injection on the CPU: one flipped limb bit in an oracle result must fail the
    bitwise comparison, and so must a flipped status bit."""
    bits = 256
    a, b = golden[f"real_{bits}_a"], golden[f"real_{bits}_b"]
    got = oracle.elementwise(bits, 2, a, b)
    want = golden[f"real_{bits}_2_out"]
    assert same(got, want)
    planted = got.copy()
    planted[17, 0] ^= 1
    assert not same(planted, want)
    planted = got.copy()
    planted[5, -1] ^= 4
    assert not same(planted, want)


ALL_WIDTHS = list(range(64, 1025, 32))


@pytest.mark.skipif(not Reference.available(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("bits", ALL_WIDTHS)
def test_oracle_matches_reference_build(oracle, bits):
    ref = Reference()
    rng = np.random.default_rng(bits)
    n = bits // 32
    cnt = 200 if bits <= 512 else 64
    a = nb.random_numbers(rng, cnt, bits, 1000, sparse_frac=0.1)
    b = nb.random_numbers(rng, cnt, bits, 1000, sparse_frac=0.1)
    c = nb.random_numbers(rng, cnt, bits, 1200, sparse_frac=0.1)
    b[::3, n] = (nb.exponent(a[::3]) - rng.integers(0, bits + 80, size=a[::3].shape[0])).astype(np.int32).view(np.uint32)
    b[1::7] = nb.negate(a[1::7])
    b[1::7, 0] ^= np.uint32(5)
    z = rng.random(cnt) < 0.05
    a[z] = 0
    for op in (0, 1, 2, 3, 7, 9, 10):
        assert same(oracle.elementwise(bits, op, a, b, c), ref.elementwise(bits, op, a, b, c)), f"op {op}"
    r = a.copy()
    r[:, n + 1] = np.abs(nb.sign(r)).astype(np.int32).view(np.uint32)
    assert same(oracle.elementwise(bits, 8, r), ref.elementwise(bits, 8, r))
    ca, cb, cc = (nb.random_complex(rng, 24, bits, 20) for _ in range(3))
    for op in (4, 5, 6, 11, 12):
        assert same(oracle.elementwise(bits, op, ca, cb, cc), ref.elementwise(bits, op, ca, cb, cc)), f"complex op {op}"
    K = 37
    A = nb.random_numbers(rng, K, bits, 200)
    B = nb.random_numbers(rng, K, bits, 200)
    cval = nb.random_numbers(rng, 1, bits, 300)[0]
    for sub in (0, 1):
        assert same(oracle.exact_dot_add(bits, cval, sub, A, 1, B, 1, K), ref.exact_dot_add(bits, cval, sub, A, 1, B, 1, K))


# ---------------------------------------------------------------- sequences vs MPFR replays
def _mp():
    return Mpfr()


def _mp_dot_sub(mp, bits, c, a, sa, b, sb, K):
    return mp.dot(bits, np.ascontiguousarray(c), 1, np.ascontiguousarray(a), sa, np.ascontiguousarray(b), sb, K)


def ref_cholesky_mpfr(mp, bits, A, n, nb_):
    """Left-looking, column by column (tests/test_cholesky.cpp:32-44): entry (i, j) is A_ij
    updated by one rounded exact dot per complete column block before j's block, then the
    in-block dot, then sqrt or a division."""
    E = bits // 32 + 3
    L = np.zeros_like(A)
    nb_ = nb_ or n
    nb_ = min(nb_, n)

    def value(i, j):
        v = A[i * n + j].copy()
        kb = j // nb_ * nb_
        for b0 in range(0, kb, nb_):
            v = _mp_dot_sub(mp, bits, v, L[i * n + b0:], 1, L[j * n + b0:], 1, nb_)
        return _mp_dot_sub(mp, bits, v, L[i * n + kb:], 1, L[j * n + kb:], 1, j - kb)

    for j in range(n):
        s = value(j, j)
        if nb.status(s) or nb.sign(s) <= 0:
            for i in range(j, n):
                for k in range(j, i + 1):
                    L[i * n + k] = 0
                    L[i * n + k, E - 1] = nb.INVALID
            return L, (j, 0 if nb.status(s) else int(nb.sign(s)), int(nb.status(s)))
        L[j * n + j] = mp.real(bits, 8, s[None])[0]
        for i in range(j + 1, n):
            L[i * n + j] = mp.real(bits, 3, value(i, j)[None], L[j * n + j][None])[0]
    return L, (n, 0, 0)


def spd_matrix(oracle, bits, n, rng):
    J = nb.random_numbers(rng, (2 * n + 1) * n, bits, 4)
    A = oracle.syrk(bits, J, 2 * n + 1, n, lower_only=False)
    for i in range(n):
        d = A[i * n + i]
        A[i * n + i] = oracle.elementwise(bits, 0, d[None], nb.power(bits, int(nb.exponent(d)) - 10))[0]
    return A


@pytest.mark.parametrize("bits,n,block", [(128, 9, 4), (96, 7, 0), (256, 6, 1), (64, 12, 5)])
def test_cholesky_oracle_vs_mpfr_replay(oracle, bits, n, block):
    mp = _mp()
    rng = np.random.default_rng(bits + n)
    A = spd_matrix(oracle, bits, n, rng)
    L, info = oracle.cholesky(bits, A, n, block)
    W, winfo = ref_cholesky_mpfr(mp, bits, A, n, block)
    assert info == winfo
    assert same(L, W)


def test_cholesky_oracle_failures(oracle):
    bits, E = 128, 7
    one, two = nb.power(bits, 0)[0], nb.power(bits, 1)[0]
    mp = _mp()
    for A, n in ((np.stack([one, one, one, one]), 2), (np.stack([one, two, two, one]), 2), (nb.negate(one[None]), 1)):
        L, info = oracle.cholesky(bits, np.ascontiguousarray(A), n, 32)
        W, winfo = ref_cholesky_mpfr(mp, bits, np.ascontiguousarray(A), n, 32)
        assert info == winfo and same(L, W)
    rng = np.random.default_rng(3)
    A = spd_matrix(oracle, bits, 8, rng)
    A[5 * 8 + 2, E - 1] = nb.INVALID
    L, info = oracle.cholesky(bits, A, 8, 3)
    W, winfo = ref_cholesky_mpfr(mp, bits, A, 8, 3)
    assert info == winfo and same(L, W)


def ref_solve_mpfr(mp, bits, L, n, X, nrhs, nb_, passes):
    """tests/test_cholesky.cpp:46-55"""
    nb_ = min(nb_ or n, n)
    X = X.copy()
    if passes & 1:
        for i in range(n):
            for c in range(nrhs):
                v = X[i * nrhs + c].copy()
                r0 = i // nb_ * nb_
                for b0 in range(0, r0, nb_):
                    v = _mp_dot_sub(mp, bits, v, L[i * n + b0:], 1, X[b0 * nrhs + c:], nrhs, nb_)
                v = _mp_dot_sub(mp, bits, v, L[i * n + r0:], 1, X[r0 * nrhs + c:], nrhs, i - r0)
                X[i * nrhs + c] = mp.real(bits, 3, v[None], L[i * n + i][None])[0]
    if passes & 2:
        for i in range(n - 1, -1, -1):
            for c in range(nrhs):
                v = X[i * nrhs + c].copy()
                r0 = i // nb_ * nb_
                r1 = min(n, r0 + nb_)
                b0 = (n - 1) // nb_ * nb_
                while b0 >= r1 and b0 > r0:
                    v = _mp_dot_sub(mp, bits, v, L[b0 * n + i:], n, X[b0 * nrhs + c:], nrhs, min(n, b0 + nb_) - b0)
                    b0 -= nb_
                if i + 1 < r1:
                    v = _mp_dot_sub(mp, bits, v, L[(i + 1) * n + i:], n, X[(i + 1) * nrhs + c:], nrhs, r1 - i - 1)
                X[i * nrhs + c] = mp.real(bits, 3, v[None], L[i * n + i][None])[0]
    return X


@pytest.mark.parametrize("passes", [1, 2, 3])
def test_solve_oracle_vs_mpfr_replay(oracle, passes):
    bits, n, nrhs, blk = 128, 9, 3, 4
    mp = _mp()
    rng = np.random.default_rng(passes)
    A = spd_matrix(oracle, bits, n, rng)
    L, info = oracle.cholesky(bits, A, n, blk)
    assert info[0] == n
    B = nb.random_numbers(rng, n * nrhs, bits, 8)
    B[4, -1] = nb.INVALID if passes == 2 else 0
    assert same(oracle.solve(bits, L, n, B, nrhs, blk, passes), ref_solve_mpfr(mp, bits, L, n, B, nrhs, blk, passes))


def _mp_complex_sequence():
    """MPFR replays of complex ops composed of real ops (tests/reference.hpp:45-55)."""
    mp = _mp()
    return mp, (lambda bits, op, x, y: mp.complex(bits, op, np.ascontiguousarray(x[None]), np.ascontiguousarray(y[None]))[0])


def test_lu4_oracle_vs_mpfr_replay(oracle):
    """tests/test_batched4.cpp:7-31: composed elimination, pivot by exact max(|re|,|im|)."""
    bits = 128
    mp, cx = _mp_complex_sequence()
    rng = np.random.default_rng(44)
    M, R = 6, 2
    A = nb.random_complex(rng, M * 16, bits, 4)
    B = nb.random_complex(rng, M * 4 * R, bits, 4)
    A[16:32:4] = 0                                   # matrix 1: zero first column
    A[32 + 8:32 + 12] = A[32:36]                     # matrix 2: duplicated rows
    X, det, st = oracle.lu4(bits, M, R, 2, A, B)
    assert st[1] == 1 and st[2] == 4
    one = np.zeros((2, bits // 32 + 3), np.uint32)
    one[0] = nb.power(bits, 0)[0]

    def mag(z):
        return z[0] if Mcmp(z[0], z[1]) >= 0 else z[1]

    def Mcmp(x, y):
        n = bits // 32
        sx, sy = int(nb.sign(x)), int(nb.sign(y))
        if not sx:
            return -1 if sy else 0
        if not sy:
            return 1
        if int(nb.exponent(x)) != int(nb.exponent(y)):
            return 1 if int(nb.exponent(x)) > int(nb.exponent(y)) else -1
        for i in range(n - 1, -1, -1):
            if x[i] != y[i]:
                return 1 if x[i] > y[i] else -1
        return 0

    for m in range(M):
        a = [A[m * 16 + i].copy() for i in range(16)]
        perm, status, swaps = [0, 1, 2, 3], 0, 0
        for k in range(4):
            piv = k
            for r in range(k + 1, 4):
                if Mcmp(mag(a[r * 4 + k]), mag(a[piv * 4 + k])) > 0:
                    piv = r
            if not nb.sign(a[piv * 4 + k][0]) and not nb.sign(a[piv * 4 + k][1]):
                status = k + 1
                break
            if piv != k:
                for c in range(4):
                    a[k * 4 + c], a[piv * 4 + c] = a[piv * 4 + c], a[k * 4 + c]
                perm[k], perm[piv] = perm[piv], perm[k]
                swaps += 1
            for r in range(k + 1, 4):
                l = cx(bits, 6, a[r * 4 + k], a[k * 4 + k])
                a[r * 4 + k] = l
                for c in range(k + 1, 4):
                    q = cx(bits, 5, l, a[k * 4 + c])
                    a[r * 4 + c] = np.stack([mp.real(bits, 1, a[r * 4 + c][0][None], q[0][None])[0],
                                             mp.real(bits, 1, a[r * 4 + c][1][None], q[1][None])[0]])
        assert st[m] == status, f"matrix {m}"
        if status:
            assert (det[m] == 0).all()
            continue
        d = a[0]
        for k in range(1, 4):
            d = cx(bits, 5, d, a[k * 5])
        if swaps & 1:
            d = nb.negate(d)
        assert same(det[m], d), f"determinant {m}"
        for j in range(R):
            y = [B[(m * 4 + perm[i]) * R + j].copy() for i in range(4)]
            for i in range(1, 4):
                for t in range(i):
                    q = cx(bits, 5, a[i * 4 + t], y[t])
                    y[i] = np.stack([mp.real(bits, 1, y[i][0][None], q[0][None])[0], mp.real(bits, 1, y[i][1][None], q[1][None])[0]])
            for i in range(3, -1, -1):
                for t in range(i + 1, 4):
                    q = cx(bits, 5, a[i * 4 + t], y[t])
                    y[i] = np.stack([mp.real(bits, 1, y[i][0][None], q[0][None])[0], mp.real(bits, 1, y[i][1][None], q[1][None])[0]])
                y[i] = cx(bits, 6, y[i], a[i * 5])
            for i in range(4):
                assert same(X[(m * 4 + i) * R + j], y[i]), f"solution {m} {i} {j}"


def test_strided_gemm_oracle_vs_mpfr_replay(oracle):
    """section9_cases.hpp:25-52: ascending k, composed cadd(sum, cmul(a, b)), accumulate from
    C, negated."""
    bits = 96
    mp, cx = _mp_complex_sequence()
    rng = np.random.default_rng(9)
    s = dict(count=2, m=3, n=4, k=5, stride_a=15, stride_b=0, stride_c=3 * 4 + 2, accumulate=True, fused=False, negative=True)
    A = nb.random_complex(rng, 30, bits, 4)
    B = nb.random_complex(rng, 20, bits, 4)
    C0 = nb.random_complex(rng, 2 * 14, bits, 4)
    got = oracle.strided_gemm(bits, True, s, A, B, C0)
    for t in range(2):
        for i in range(3):
            for j in range(4):
                z = C0[t * 14 + i * 4 + j]
                for k in range(5):
                    z = cx(bits, 4, z, cx(bits, 5, A[t * 15 + i * 5 + k], B[k * 4 + j]))
                assert same(got[t * 14 + i * 4 + j], nb.negate(z)), (t, i, j)
    assert same(got[12:14], C0[12:14])               # padding between outputs kept


@pytest.mark.parametrize("bits", [64, 128, 256, 480, 1024])
def test_oracle_fused_three_term_cases(oracle, bits):
    """Adversarial cfma operands (tests/fused_cases.py): the oracle agrees with an MPFR sum of the two
    exact products and the addend rounded once per component, and with the reference build."""
    from fused_cases import dot2_cases
    rng = np.random.default_rng(4242 + bits)
    a, b, c = dot2_cases(rng, bits, 160)
    got = oracle.elementwise(bits, 11, a, b, c)
    mp = _mp()
    re = lambda z: np.ascontiguousarray(z[:, 0])
    im = lambda z: np.ascontiguousarray(z[:, 1])
    want_re = mp.dot2_add(bits, re(a), re(b), np.ascontiguousarray(nb.negate(im(a))), im(b), re(c))
    want_im = mp.dot2_add(bits, re(a), im(b), im(a), re(b), im(c))
    assert same(np.ascontiguousarray(got[:, 0]), want_re), "re vs MPFR"
    assert same(np.ascontiguousarray(got[:, 1]), want_im), "im vs MPFR"
    if Reference.available():
        assert same(got, Reference().elementwise(bits, 11, a, b, c)), "vs reference build"


@pytest.mark.skipif(not Reference.available(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("bits", [96, 256, 640])
def test_sequence_oracles_vs_reference_build(oracle, bits):
    """Segmented dots and recurrences of the oracle equal the same chains stepped with the reference's own
    fma / cfma / cmul / cadd (its core.hpp, built from its sources)."""
    ref = Reference()
    rng = np.random.default_rng(bits + 77)
    seg, ln = 12, 9
    for cx in (False, True):
        make = (lambda c: nb.random_complex(rng, c, bits, 30)) if cx else (lambda c: nb.random_numbers(rng, c, bits, 30, sparse_frac=0.1))
        a, b = make(seg * ln), make(seg * ln)
        for shared in (False, True):
            got = oracle.segmented_dot(bits, cx, seg, ln, shared, a, b)
            s = np.zeros_like(got)
            for k in range(ln):
                x = np.ascontiguousarray(a.reshape(seg, ln, *a.shape[1:])[:, k])
                y = np.ascontiguousarray(np.broadcast_to(b[k], x.shape) if shared else b.reshape(seg, ln, *b.shape[1:])[:, k])
                s = ref.elementwise(bits, 11 if cx else 9, x, y, np.ascontiguousarray(s))
            assert same(got, s), f"segmented dot complex={cx} shared={shared}"
    count, steps, spw = 16, 5, 2
    seeds = nb.random_complex(rng, 4 * count, bits, 3)
    weights = nb.random_complex(rng, steps * 4 * (count // spw), bits, 2)
    got = oracle.recurrence(bits, seeds, weights, count, steps, spw)
    q = [np.ascontiguousarray(seeds[j * count:(j + 1) * count]) for j in range(4)]
    G = count // spw
    for t in range(steps):
        s = np.zeros_like(q[0])
        for j in range(4):
            w = np.ascontiguousarray(weights[(t * 4 + j) * G:(t * 4 + j + 1) * G][np.arange(count) // spw])
            s = ref.elementwise(bits, 4, s, ref.elementwise(bits, 5, w, q[j]))
        q = q[1:] + [s]
    assert same(got, q[3]), "recurrence"
