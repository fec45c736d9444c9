"""CPU: pin the oracle's Householder QR (lf_oracle.c: the column order of the reference's tests/test_qr.cpp with
the term sets of its library's blocked sequence, src/linalg.mm:488-790) before the GPU factor is checked against it.

* golden factors (tests/golden/qr_golden.npz) from the library's blocked right-looking sequence evaluated
  with the reference's own arithmetic (oracle/_ref's ref_qr_blocked);
* the same comparison on fresh inputs of every matrix kind and special case, when oracle/_ref is present;
* the fixtures' expected ranks (zero columns, statuses, dependent columns found with a rank test);
* column pivoting: a full-rank status-free factor equals the unpivoted factor of A P, and the pivoting
  fixtures' ranks, tie-breaking and norm recomputations;
* least squares and Q applications: Q^T Q B and Q Q^T B return to B up to rounding, and the solve of a
  consistent system returns its solution up to rounding;
* a planted mistake in an oracle factor is caught.
"""
import os

import numpy as np
import pytest

from limbforge_b200 import numbers as nb
from oracle.oracle import Reference
from tests import qr_cases as qc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def qr_golden():
    return np.load(os.path.join(ROOT, "tests", "golden", "qr_golden.npz"))


def same_factor(f, g):
    return all(f[k].shape == g[k].shape and bool((f[k] == g[k]).all()) for k in ("R", "V", "T", "tau")) and \
        (f["rank"], f["reason"], f["status"]) == (g["rank"], g["reason"], g["status"])


def test_qr_oracle_matches_golden(oracle, qr_golden):
    for i in range(int(qr_golden["count"])):
        meta = qr_golden[f"c{i}_meta"]
        bits, m, n, block, rank_bits = (int(x) for x in meta[:5])
        f = oracle.qr(bits, qr_golden[f"c{i}_A"], m, n, block, rank_bits)
        label = str(qr_golden[f"c{i}_label"])
        for k in ("R", "V", "T", "tau"):
            assert (f[k] == qr_golden[f"c{i}_{k}"]).all(), f"{label}: {k}"
        assert (f["rank"], f["reason"], f["status"]) == tuple(int(x) for x in meta[5:]), label


@pytest.mark.skipif(not Reference.available(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("bits", [64, 224, 256, 384])
def test_qr_oracle_matches_reference_blocked(oracle, bits):
    ref = Reference()
    rng = np.random.default_rng(5151 + bits)
    shapes = [(1, 1, "moderate", 32), (3, 2, "qsc", 32), (33, 7, "graded", 32), (64, 32, "wide", 16), (70, 40, "spread", 7),
              (40, 40, "extreme", 0), (31, 17, "triangular", 16), (50, 33, "dependent", 16), (49, 33, "qsc", 32)]
    for m, n, kind, block in shapes:
        A = qc.matrix(bits, m, n, kind, rng)
        assert same_factor(oracle.qr(bits, A, m, n, block), ref.qr_blocked(bits, A, m, n, block)), f"{kind} {m}x{n} block {block}"
    if bits == 256:
        for label, A, m, n, rank_bits, _ in qc.special_cases(bits, rng):
            for block in (16, 7):
                got, want = oracle.qr(bits, A, m, n, block, rank_bits), ref.qr_blocked(bits, A, m, n, block, rank_bits)
                assert same_factor(got, want), f"{label} block {block}"


def test_qr_oracle_fixture_ranks(oracle):
    bits = 256
    rng = np.random.default_rng(77)
    for label, A, m, n, rank_bits, expect in qc.special_cases(bits, rng):
        f = oracle.qr(bits, A, m, n, 16, rank_bits)
        if expect is not None:
            assert f["rank"] == expect, f"{label}: rank {f['rank']}, fixture expects {expect}"
        if f["rank"] == n:
            assert f["reason"] == 0
    # the entry 2^-999999995 leaves the exponent range when v is scaled: tau carries exponent_overflow
    cases = {c[0]: c for c in qc.special_cases(bits, rng)}
    label, A, m, n, rank_bits, _ = cases["tiny entry in column 0"]
    f = oracle.qr(bits, A, m, n, 16, rank_bits)
    assert nb.status(f["tau"][:1])[0] == nb.EXPONENT_OVERFLOW
    # reflector 3 carries the status: R's rows 0..2 in later columns see it (the library's term sets)
    label, A, m, n, rank_bits, _ = cases["tiny entry in column 3"]
    f = oracle.qr(bits, A, m, n, 16, rank_bits)
    assert nb.status(f["tau"][3:4])[0] == nb.EXPONENT_OVERFLOW and f["rank"] == 4 and f["reason"] == 3
    assert (nb.status(f["R"].reshape(n, n, -1)[0, 5:]) == nb.EXPONENT_OVERFLOW).all()


def permuted(A, m, n, perm):
    return A.reshape(m, n, -1)[:, perm, :].reshape(m * n, -1).copy()


def test_qr_pivoted_equals_unpivoted_of_permuted(oracle):
    bits = 256
    rng = np.random.default_rng(99)
    for m, n, kind in [(1, 1, "moderate"), (5, 3, "qsc"), (33, 7, "graded"), (60, 30, "qsc"), (64, 32, "wide"), (70, 40, "spread")]:
        A = qc.matrix(bits, m, n, kind, rng)
        for block in (16, 7, 0):
            f = oracle.qr(bits, A, m, n, block, 0, pivot=True)
            assert f["rank"] == n and sorted(f["perm"]) == list(range(n))
            u = oracle.qr(bits, permuted(A, m, n, f["perm"]), m, n, block)
            assert same_factor(f, u), f"{kind} {m}x{n} block {block}"
            # |r_jj| nonincreasing up to rounding: exponents never grow by more than one binade
            e = [int(nb.exponent(f["R"][j * n + j][None])[0]) for j in range(n)]
            assert all(e[j + 1] <= e[j] + 1 for j in range(n - 1))


def test_qr_pivoted_fixtures(oracle):
    bits = 256
    N = bits // 32
    rng = np.random.default_rng(7)
    f = oracle.qr(bits, qc.matrix(bits, 41, 7, "dependent", rng), 41, 7, 16, bits // 2, pivot=True)
    assert f["rank"] == 5 and f["reason"] == 2
    f = oracle.qr(bits, qc.matrix(bits, 90, 40, "dependent", rng), 90, 40, 16, bits // 2, pivot=True)
    assert f["rank"] == 38
    A = qc.matrix(bits, 30, 12, "moderate", rng)
    A[2::12] = 0
    A[7::12] = 0
    f = oracle.qr(bits, A, 30, 12, 16, 0, pivot=True)
    assert f["rank"] == 10 and f["reason"] == 1 and set(f["perm"][10:]) == {2, 7}
    A = qc.matrix(bits, 25, 9, "moderate", rng)
    for r in range(25):
        A[r * 9 + 6] = A[r * 9 + 2]
        A[r * 9 + 8] = A[r * 9 + 2]
    f = oracle.qr(bits, A, 25, 9, 16, bits // 2, pivot=True)
    assert f["rank"] == 7 and f["perm"].index(2) < f["perm"].index(6) < f["perm"].index(8)
    A = qc.matrix(bits, 25, 10, "moderate", rng)
    A[7 * 10 + 4, N + 2] = nb.INVALID
    f = oracle.qr(bits, A, 25, 10, 16, 0, pivot=True)
    assert (f["rank"], f["reason"], f["status"]) == (0, 3, nb.INVALID) and f["perm"][0] == 4
    # nearly parallel columns: downdated norms collapse and are recomputed
    A = qc.matrix(bits, 80, 20, "moderate", rng)
    for j in (5, 13):
        t = nb.random_numbers(rng, 80, bits, 4)
        t[:, N] = (nb.exponent(t) - (bits // 4 + 10)).astype(np.int32).view(np.uint32)
        A[j::20] = oracle.elementwise(bits, 0, np.ascontiguousarray(A[j - 1::20]), t)
    f = oracle.qr(bits, A, 80, 20, 16, 0, pivot=True)
    assert f["recomputed"] > 0


def close(x, y, bits, lost):
    """every entry of x within 2^-(bits - lost) of the largest |y| (exact rationals)"""
    fx = [nb.to_fraction(v) for v in x]
    fy = [nb.to_fraction(v) for v in y]
    scale = max(abs(v) for v in fy)
    return all(abs(a - b) <= scale / 2 ** (bits - lost) for a, b in zip(fx, fy))


def test_qr_solve_and_apply_round_trip(oracle):
    bits = 256
    rng = np.random.default_rng(11)
    m, n, nrhs = 40, 18, 3
    for pivot in (False, True):
        A = qc.matrix(bits, m, n, "moderate", rng)
        f = oracle.qr(bits, A, m, n, 8, 0, pivot=pivot)
        B = qc.rhs(bits, m, nrhs, rng)
        back = oracle.qr_apply(f, oracle.qr_apply(f, B, nrhs, True), nrhs, False)
        assert close(back, B, bits, 16)
        # a consistent system: B = A X0 (exact products rounded once), the solve returns X0 up to rounding
        X0 = nb.random_numbers(rng, n * nrhs, bits, 2)
        Bc = np.zeros((m * nrhs, bits // 32 + 3), dtype=np.uint32)
        for r in range(m):
            for c in range(nrhs):
                Bc[r * nrhs + c] = oracle.exact_dot_add(bits, None, False, A[r * n:], 1, X0[c:], nrhs, n)
        X = oracle.qr_solve(f, Bc, nrhs)
        assert close(X, X0, bits, 32)


def test_qr_rank_deficient_solve_is_invalid(oracle):
    bits = 256
    rng = np.random.default_rng(12)
    A = qc.zero_column(qc.matrix(bits, 20, 9, "moderate", rng), 20, 9, 3)
    f = oracle.qr(bits, A, 20, 9, 16)
    X = oracle.qr_solve(f, qc.rhs(bits, 20, 2, rng), 2)
    assert (nb.status(X) == nb.INVALID).all() and (nb.sign(X) == 0).all()


def test_qr_planted_mistake_is_caught(oracle, qr_golden):
    meta = qr_golden["c1_meta"]
    bits, m, n, block, rank_bits = (int(x) for x in meta[:5])
    f = oracle.qr(bits, qr_golden["c1_A"], m, n, block, rank_bits)
    f["R"][5, 0] ^= 1
    assert not (f["R"] == qr_golden["c1_R"]).all()


# ---- complex QR (lf_oracle.c lfo_qr_complex: the library's complex sequence, linalg_complex.mm)
def test_qr_complex_real_input_is_the_real_qr(oracle):
    """The reference test's own cross-check (tests/test_qr_complex.cpp:7): a real matrix gives the real QR bit for bit
    in the real parts and zero imaginary parts, unpivoted and pivoted, with the same solves and Q applications."""
    bits = 256
    w = bits // 32 + 3
    rng = np.random.default_rng(21)
    for m, n, kind, block in [(33, 7, "graded", 32), (40, 21, "qsc", 8), (50, 33, "spread", 16), (20, 9, "moderate", 4)]:
        A = qc.matrix(bits, m, n, kind, rng)
        Ac = np.zeros((m * n, 2, w), np.uint32)
        Ac[:, 0] = A
        for pivot in (False, True):
            fc, fr = oracle.qr_complex(bits, Ac, m, n, block, 0, pivot), oracle.qr(bits, A, m, n, block, 0, pivot)
            for k in ("R", "V", "tau", "T"):
                assert (fc[k][:, 0] == fr[k]).all() and (fc[k][:, 1] == 0).all(), f"{kind} {k} pivot={pivot}"
            assert fc["perm"] == fr["perm"] and fc["rank"] == fr["rank"]
            B = qc.rhs(bits, m, 3, rng)
            Bc = np.zeros((m * 3, 2, w), np.uint32)
            Bc[:, 0] = B
            X = oracle.qr_complex_solve(fc, Bc, 3)
            assert (X[:, 0] == oracle.qr_solve(fr, B, 3)).all() and (X[:, 1] == 0).all()
            for qt in (True, False):
                C1 = oracle.qr_complex_apply(fc, Bc, 3, qt)
                assert (C1[:, 0] == oracle.qr_apply(fr, B, 3, qt)).all() and (C1[:, 1] == 0).all()


def cfrac(z):
    return [(nb.to_fraction(v[0]), nb.to_fraction(v[1])) for v in z]


def ccheck(x, y, bits, lost):
    fx, fy = cfrac(x), cfrac(y)
    scale = max(max(abs(a), abs(b)) for a, b in fy)
    return all(abs(a - c) <= scale / 2 ** (bits - lost) and abs(b - d) <= scale / 2 ** (bits - lost) for (a, b), (c, d) in zip(fx, fy))


def test_qr_complex_properties(oracle):
    bits = 256
    N = bits // 32
    rng = np.random.default_rng(22)
    m, n, nrhs = 30, 12, 2
    for pivot in (False, True):
        A = qc.complex_matrix(bits, m, n, "moderate", rng)
        f = oracle.qr_complex(bits, A, m, n, 5, 0, pivot)
        assert f["rank"] == n
        assert (f["R"].reshape(n, n, 2, -1)[np.arange(n), np.arange(n), 1] == 0).all()      # real diagonal
        B = qc.complex_rhs(bits, m, nrhs, rng)
        back = oracle.qr_complex_apply(f, oracle.qr_complex_apply(f, B, nrhs, True), nrhs, False)
        assert ccheck(back, B, bits, 16)
        # a consistent system B = A X0 (each component one exact dot), solved back to X0 up to rounding
        X0 = np.zeros((n * nrhs, 2, N + 3), np.uint32)
        X0[:, 0] = nb.random_numbers(rng, n * nrhs, bits, 2)
        X0[:, 1] = nb.random_numbers(rng, n * nrhs, bits, 2)
        Bc = np.zeros((m * nrhs, 2, N + 3), np.uint32)
        for r in range(m):
            a = np.ascontiguousarray(A[r * n:(r + 1) * n].reshape(2 * n, -1))
            for c in range(nrhs):
                x = X0[c::nrhs][:n]
                xr = np.ascontiguousarray(np.stack([x[:, 0], nb.negate(x[:, 1])], 1).reshape(2 * n, -1))
                xi = np.ascontiguousarray(np.stack([x[:, 1], x[:, 0]], 1).reshape(2 * n, -1))
                Bc[r * nrhs + c, 0] = oracle.exact_dot_add(bits, None, False, a, 1, xr, 1, 2 * n)
                Bc[r * nrhs + c, 1] = oracle.exact_dot_add(bits, None, False, a, 1, xi, 1, 2 * n)
        assert ccheck(oracle.qr_complex_solve(f, Bc, nrhs), X0, bits, 40)
        if pivot:
            AP = A.reshape(m, n, 2, -1)[:, f["perm"]].reshape(m * n, 2, -1).copy()
            u = oracle.qr_complex(bits, AP, m, n, 5)
            for k in ("R", "V", "tau", "T"):
                assert (u[k] == f[k]).all(), f"pivoted complex vs A P: {k}"


def test_qr_complex_fixture_ranks(oracle):
    bits = 256
    N = bits // 32
    rng = np.random.default_rng(23)
    A = qc.complex_matrix(bits, 20, 9, "moderate", rng)
    A[3::9] = 0
    assert oracle.qr_complex(bits, A, 20, 9, 4)["rank"] == 3
    A = qc.complex_matrix(bits, 25, 10, "moderate", rng)
    A[7 * 10 + 4, 1, N + 2] = nb.INVALID
    f = oracle.qr_complex(bits, A, 25, 10, 4)
    assert (f["rank"], f["reason"], f["status"]) == (4, 3, nb.INVALID)
    f = oracle.qr_complex(bits, qc.complex_matrix(bits, 41, 7, "dependent", rng), 41, 7, 16, bits // 2)
    assert f["rank"] == 3 and f["reason"] == 2
    f = oracle.qr_complex(bits, qc.complex_matrix(bits, 41, 7, "dependent", rng), 41, 7, 16, bits // 2, True)
    assert f["rank"] == 5
    # a column that is purely imaginary on the diagonal and zero below still reflects (tau complex)
    A = qc.complex_matrix(bits, 6, 3, "moderate", rng)
    A[0::3] = 0
    A[0, 1] = nb.power(bits, 3)[0]
    f = oracle.qr_complex(bits, A, 6, 3, 2)
    assert f["rank"] == 3 and nb.sign(f["tau"][0, 1][None])[0] != 0
