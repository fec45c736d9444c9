"""Matrix fixtures for the Householder QR tests, following the kinds and special cases of the reference's
tests/test_qr.cpp:150-162 (moderate, qsc, wide, spread, graded, dependent, upper triangular, extreme spread) and
:174-207 (zero columns, statuses, exactly dependent columns with a rank test, extreme spreads, an entry far below
the others, the augmented Levenberg-Marquardt matrix), regenerated with numpy seeds."""
import numpy as np

from limbforge_b200 import numbers as nb

KINDS = ["moderate", "qsc", "wide", "spread", "graded", "dependent", "triangular", "extreme"]


def matrix(bits, m, n, kind, rng):
    """m x n row-major matrix, shape (m * n, N + 3)."""
    w = bits // 32 + 3
    N = bits // 32
    A = np.zeros((m * n, w), dtype=np.uint32)
    span = {"qsc": 15, "spread": 400, "extreme": 3000}.get(kind, 4)
    for c in range(n):
        scale = (int(rng.integers(-60, 61)) if kind == "qsc" else int(rng.integers(-300, 301)) if kind == "wide"
                 else (20 if c % 2 else -20) if kind == "graded" else 0)
        col = nb.random_numbers(rng, m, bits, span)
        col[:, N] = (nb.exponent(col) + scale).astype(np.int32).view(np.uint32)
        if kind == "qsc":
            col[rng.integers(0, 4, size=m) == 0] = 0
        if kind == "triangular":
            col[c + 1:] = 0
        A[c::n] = col
        if kind == "qsc" and c % 17 == 5:
            r = int(rng.integers(0, m))
            if nb.sign(A[r * n + c][None])[0]:
                A[r * n + c, N] = np.int32(scale - 150).view(np.uint32)
    if kind == "dependent" and n >= 3:
        for r in range(m):
            A[r * n + n - 1] = A[r * n + 1]
            A[r * n + n // 2] = nb.negate(A[r * n][None])[0]
    return A


def rhs(bits, m, nrhs, rng):
    B = nb.random_numbers(rng, m * nrhs, bits, 8)
    B[rng.integers(0, 11, size=m * nrhs) == 0] = 0
    return B


def zero_column(A, m, n, c):
    A[c::n] = 0
    return A


def special_cases(bits, rng):
    """(label, A, m, n, rank_bits, expected rank or None) of the reference's special cases."""
    N = bits // 32
    out = []
    A = zero_column(matrix(bits, 20, 9, "moderate", rng), 20, 9, 3)
    out.append(("zero column 3", A, 20, 9, 0, 3))
    out.append(("zero matrix", np.zeros((12, N + 3), dtype=np.uint32), 4, 3, 0, 0))
    A = zero_column(matrix(bits, 40, 20, "qsc", rng), 40, 20, 0)
    out.append(("zero column 0", A, 40, 20, 0, 0))
    out.append(("upper triangular square", matrix(bits, 12, 12, "triangular", rng), 12, 12, 0, 12))
    out.append(("upper triangular tall", matrix(bits, 30, 18, "triangular", rng), 30, 18, 0, 18))
    A = matrix(bits, 25, 10, "moderate", rng); A[7 * 10 + 4, N + 2] = nb.INVALID
    out.append(("status at (7,4)", A, 25, 10, 0, 4))
    A = matrix(bits, 25, 10, "moderate", rng); A[20 * 10 + 0, N + 2] = nb.EXPONENT_OVERFLOW
    out.append(("status at (20,0)", A, 25, 10, 0, 0))
    A = zero_column(matrix(bits, 25, 10, "moderate", rng), 25, 10, 6); A[3 * 10 + 8, N + 2] = nb.INVALID
    out.append(("zero column 6, status in 8", A, 25, 10, 0, 6))
    A = zero_column(matrix(bits, 40, 30, "moderate", rng), 40, 30, 0); A[5 * 30 + 20, N + 2] = nb.INVALID
    out.append(("zero column 0, status in 20", A, 40, 30, 0, 0))
    A = matrix(bits, 41, 7, "dependent", rng)
    out.append(("dependent, no rank test", A, 41, 7, 0, None))
    out.append(("dependent, rank_bits", A, 41, 7, bits // 2, 3))
    out.append(("dependent 90x40, rank_bits", matrix(bits, 90, 40, "dependent", rng), 90, 40, bits // 2, 20))
    out.append(("extreme spread", matrix(bits, 300, 24, "extreme", rng), 300, 24, 0, None))
    A = matrix(bits, 150, 12, "moderate", rng)
    for r in range(150):
        if nb.sign(A[r * 12][None])[0]:
            A[r * 12, N] = np.int32(int(np.int32(A[r * 12, N].view(np.int32))) + 10).view(np.uint32)
    A[77 * 12] = nb.power(bits, -999999995)[0]
    out.append(("tiny entry in column 0", A, 150, 12, 0, None))
    # the same in column 3 with zeros beside it in columns 0..2: reflector 3 carries the status; the rows above it
    # see it in every later rounding that applies the block (the library's term sets)
    A = matrix(bits, 60, 12, "moderate", rng)
    A[37 * 12:37 * 12 + 3] = 0
    A[37 * 12 + 3] = nb.power(bits, -999999995)[0]
    out.append(("tiny entry in column 3", A, 60, 12, 0, 4))
    return out


def augmented(bits, J, m, n, d):
    """[J; diag(d)] ((m + n) x n)."""
    w = bits // 32 + 3
    S = np.zeros(((m + n) * n, w), dtype=np.uint32)
    S[:m * n] = J
    for i in range(n):
        S[(m + i) * n + i] = d[i]
    return S


def complex_matrix(bits, m, n, kind, rng):
    """m x n complex row-major matrix, shape (m * n, 2, N + 3): independent real and imaginary parts of `kind`
    (the dependent kind keeps its dependence: both parts repeat column 1 in the last column and negate column 0
    in column n // 2)."""
    w = bits // 32 + 3
    A = np.zeros((m * n, 2, w), dtype=np.uint32)
    A[:, 0] = matrix(bits, m, n, kind, rng)
    A[:, 1] = matrix(bits, m, n, kind, rng)
    if kind == "dependent" and n >= 3:
        for r in range(m):
            A[r * n + n - 1] = A[r * n + 1]
            A[r * n + n // 2, 0] = nb.negate(A[r * n, 0][None])[0]
            A[r * n + n // 2, 1] = nb.negate(A[r * n, 1][None])[0]
    return A


def complex_rhs(bits, m, nrhs, rng):
    w = bits // 32 + 3
    B = np.zeros((m * nrhs, 2, w), dtype=np.uint32)
    B[:, 0] = rhs(bits, m, nrhs, rng)
    B[:, 1] = rhs(bits, m, nrhs, rng)
    return B
