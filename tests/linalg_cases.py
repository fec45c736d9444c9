"""Matrix fixtures for the exact-product and factorization tests, following the kinds of the
reference's tests/test_linalg.cpp:71-106 (moderate, wide, cancel, sparse, qsc, ties, saturated),
old-entry kinds for updates (test_linalg.cpp:126-136) and SPD kinds of test_cholesky.cpp:57-78,
regenerated with numpy seeds."""
import numpy as np

from limbforge_b200 import numbers as nb

KINDS = ["moderate", "wide", "cancel", "sparse", "qsc", "ties", "saturated"]


def power(bits, e, s=1):
    return nb.power(bits, int(e), s)[0]


def matrix(bits, rows, cols, kind, rng):
    n = bits // 32
    A = np.zeros((rows * cols, n + 3), dtype=np.uint32)

    def at(r, c):
        return r * cols + c
    for c in range(cols):
        scale = int(rng.integers(-1000, 1001)) if kind == "wide" else int(rng.integers(-60, 61)) if kind == "qsc" else 0
        span = 15 if kind == "qsc" else 30 if kind == "wide" else 4
        col = nb.random_numbers(rng, rows, bits, span)
        col[:, n] = (nb.exponent(col) + scale + (-10 if kind == "qsc" else 0)).astype(np.int32).view(np.uint32)
        p0 = 3 if kind == "sparse" else 4 if kind == "qsc" else 10
        col[rng.integers(0, p0, size=rows) == 0] = 0
        A[[at(r, c) for r in range(rows)]] = col
        if kind == "wide":
            r = int(rng.integers(0, rows))
            m9 = c % 9
            if m9 in (1, 2):
                A[at(r, c), n] = np.uint32(np.int32(scale - 100 - int(rng.integers(0, 350))).view(np.uint32))
            elif m9 == 3:
                A[at(r, c), n] = np.int32(scale - 5000).view(np.uint32)
            elif m9 == 4:
                for q in range(0, rows, 2):
                    A[at(q, c), n] = np.int32(scale - 70 * (q // 2 % 5)).view(np.uint32)
            elif m9 == 7:
                for q in range(0, rows, 2):
                    A[at(q, c), n] = np.int32(scale - 100 * (q // 2 % 3)).view(np.uint32)
            elif m9 == 8:
                for q in range(1, rows, 2):
                    A[at(q, c), n] = np.int32(scale - 90 * (q // 2 % 4)).view(np.uint32)
            elif m9 == 5:
                A[at(r, c), n] = np.int32(600000000).view(np.uint32)
            elif m9 == 6:
                for q in range(rows):
                    A[at(q, c), n] = np.int32(-600000000 + q % 5).view(np.uint32)
            zero = (nb.sign(A[[at(q, c) for q in range(rows)]]) == 0)
            for q in np.nonzero(zero)[0]:
                A[at(q, c)] = 0                                        # keep zeros canonical
        if kind == "qsc" and c % 17 == 5:
            r = int(rng.integers(0, rows))
            if nb.sign(A[at(r, c)]):
                A[at(r, c), n] = np.int32(scale - 150).view(np.uint32)
        if kind == "sparse":
            if c % 11 == 3:
                for r in range(rows):
                    A[at(r, c)] = 0
            if c % 13 == 7:
                A[at(int(rng.integers(0, rows)), c), n + 2] = nb.INVALID if rng.integers(0, 2) else nb.EXPONENT_OVERFLOW
    if kind == "cancel":
        h = rows // 2
        for c in range(0, cols - 1, 2):
            for r in range(h):
                A[at(r + h, c)] = A[at(r, c)]
                A[at(r, c + 1)] = A[at(r, c)]
                A[at(r + h, c + 1)] = nb.negate(A[at(r, c)][None])[0]
            if rows % 2 and c % 4 == 0:
                A[at(rows - 1, c)] = power(bits, -400 - c % 3)
                A[at(rows - 1, c + 1)] = power(bits, -401, 1 if c % 8 else -1)
            if c % 6 == 2 and h:
                A[at(0, c + 1), 0] ^= 1
    if kind == "ties" and rows >= 4:
        p = [1, bits // 2, bits // 2 - 1, bits // 2 + 1, bits - 1, 3]
        for c in range(cols):
            u = power(bits, 0)
            if c % 3 == 1:
                u[0] |= 1
            if c % 5 == 4:
                u = nb.negate(u[None])[0]
            for r in range(rows):
                A[at(r, c)] = 0
            A[at(0, c)] = u
            A[at(1, c)] = power(bits, -p[c % 6])
            A[at(2, c)] = power(bits, 200 + c % 2)
            A[at(3, c)] = power(bits, 200 + c % 2, 1 if c % 4 < 2 else -1)
    if kind == "saturated":
        for r in range(rows):
            for c in range(cols):
                x = power(bits, -9 if (c % 5 == 4 and r % 2) else 0)
                x[:n] = 0xffffffff
                A[at(r, c)] = x
    return A


def old_entries(bits, P, rng):
    """Old C for updates: RN(product) itself, the same far above/below, zeros, statuses, random."""
    n = bits // 32
    C = np.zeros_like(P)
    for q in range(P.shape[0]):
        p = P[q]
        sgn = int(nb.sign(p))
        k = int(rng.integers(0, 8))
        if k in (0, 1):
            C[q] = p
        elif k == 2:
            C[q] = p.copy()
            if sgn:
                C[q, n] = np.int32(int(nb.exponent(p)) + bits + 2).view(np.uint32)
        elif k == 3:
            if sgn:
                C[q] = nb.negate(p[None])[0]
                C[q, n] = np.int32(int(nb.exponent(p)) - bits - 5).view(np.uint32)
        elif k == 4:
            C[q] = 0
        elif k == 5:
            C[q] = power(bits, 9)
            C[q, n + 2] = nb.INVALID if rng.integers(0, 2) else nb.DIVISION_BY_ZERO
        else:
            x = nb.random_numbers(rng, 1, bits, 3 if sgn else 300)[0]
            if sgn:
                x[n] = np.int32(int(nb.exponent(x)) + int(nb.exponent(p))).view(np.uint32)
            C[q] = x
    return C


def spd(oracle, bits, n, kind, rng):
    """A = J^T J + damping (test_cholesky.cpp:57-78), banded or rank-deficient variants."""
    nn = bits // 32
    if kind == "banded":
        A = np.zeros((n * n, nn + 3), dtype=np.uint32)
        for i in range(n):
            d = nb.random_numbers(rng, 1, bits, 0)[0]
            nb.set_fields(d, 3, 1)
            A[i * n + i] = d
            for dd in (1, 3):
                if dd <= i:
                    x = nb.random_numbers(rng, 1, bits, 0)[0]
                    x[nn] = np.int32(-1).view(np.uint32)
                    A[i * n + i - dd] = x
                    A[(i - dd) * n + i] = x
        return A
    m = 2 * n + 1
    J = np.zeros((m * n, nn + 3), dtype=np.uint32)
    for c in range(n):
        scale = int(rng.integers(-60, 61)) if kind == "qsc" else int(rng.integers(-300, 301)) if kind == "wide" else \
            (20 if c % 2 else -20) if kind == "graded" else 0
        col = nb.random_numbers(rng, m, bits, 15 if kind == "qsc" else 4)
        col[:, nn] = (nb.exponent(col) + scale).astype(np.int32).view(np.uint32)
        if kind == "qsc":
            col[rng.integers(0, 4, size=m) == 0] = 0
        J[np.arange(m) * n + c] = col
    if kind == "rank_deficient" and n >= 3:
        for r in range(m):
            J[r * n + n - 1] = J[r * n + 1]
            J[r * n + n // 2] = nb.negate(J[r * n][None])[0]
    A = oracle.syrk(bits, J, m, n, lower_only=False)
    if kind != "rank_deficient":
        for i in range(n):
            a = A[i * n + i]
            if nb.sign(a):
                A[i * n + i] = oracle.elementwise(bits, 0, a[None].copy(), power(bits, int(nb.exponent(a)) - 10)[None])[0]
    return A


def rhs(bits, n, nrhs, rng):
    B = nb.random_numbers(rng, n * nrhs, bits, 8)
    B[rng.integers(0, 11, size=n * nrhs) == 0] = 0
    return B
