"""ctypes front end of the CPU checkers (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this
module, and only to check or time against it.  The product package never does.

Arrays are numpy ``uint32`` arrays holding the reference's element layout
(include/limbforge/core.hpp:23-34): ``[..., N+3]`` words per real element (N limbs,
exponent, sign, status) and ``[..., 2, N+3]`` per complex element (re, im).

Three checkers are exposed:

* ``Oracle``   -- lf_oracle.c, the C restatement (exact integers, one RNE rounding).
* ``Reference`` -- oracle/_ref/libref.so, the reference's own core.hpp/exact_dot_add
  compiled from its sources (absent where the reference checkout is absent).
* ``Mpfr``     -- mpfr_shim.c, independent MPFR replays as in tests/reference.hpp.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


def build(reference: str | None = None) -> None:
    """Compile the checkers in place (make -C oracle)."""
    cmd = ["make", "-s", "-C", HERE]
    if reference:
        cmd.append(f"REFERENCE={reference}")
    subprocess.run(cmd, check=True)


def _load(name: str) -> C.CDLL:
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        build()
    return C.CDLL(path)


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


class Oracle:
    """The C restatement of the reference's arithmetic contract."""

    def __init__(self) -> None:
        lib = _load("liblf_oracle.so")
        V, S, I, L = C.c_void_p, C.c_size_t, C.c_int, C.c_long
        lib.lfo_elementwise.argtypes = [I, I, V, V, V, V, S, S, S, S, S]
        lib.lfo_mul_chain.argtypes = [I, V, V, S, V, S]
        lib.lfo_exact_dot_add_bits.argtypes = [I, V, I, V, L, V, L, S, V]
        lib.lfo_gemm_rows.argtypes = [I, I, V, V, S, S, S, V, I, S, S]
        lib.lfo_syrk_rows.argtypes = [I, V, S, S, V, I, I, S, S]
        lib.lfo_cholesky.argtypes = [I, V, S, V, S, C.POINTER(C.c_long)]
        lib.lfo_solve.argtypes = [I, V, S, V, S, S, I]
        lib.lfo_lu4.argtypes = [I, S, C.c_uint, I, V, V, V, V, V]
        lib.lfo_strided_gemm.argtypes = [I, I, S, S, S, S, S, S, S, I, I, I, V, V, V]
        lib.lfo_dot2_add.argtypes = [I, V, V, V, V, V, V]
        lib.lfo_cast.argtypes = [I, I, I, V, V, S]
        lib.lfo_tree_sum.argtypes = [I, I, V, S, V]
        lib.lfo_segmented_dot.argtypes = [I, I, S, S, I, V, V, V]
        lib.lfo_recurrence.argtypes = [I, V, V, V, S, C.c_uint, C.c_uint]
        lib.lfo_qr.argtypes = [I, V, S, S, S, I, V, V, V, V, C.POINTER(C.c_long)]
        lib.lfo_qr_pivoted.argtypes = [I, V, S, S, S, I, V, V, V, V, C.POINTER(C.c_size_t), C.POINTER(C.c_long)]
        lib.lfo_qr_apply.argtypes = [I, S, S, S, S, V, V, V, S, I]
        lib.lfo_qr_solve.argtypes = [I, S, S, S, C.POINTER(C.c_long), C.POINTER(C.c_size_t), V, V, V, V, S, V]
        lib.lfo_exact_gemm4.argtypes = [I, I, S, S, S, S, I, I, V, V, V]
        lib.lfo_qr_complex.argtypes = [I, V, S, S, S, I, I, V, V, V, V, C.POINTER(C.c_size_t), C.POINTER(C.c_long)]
        lib.lfo_qr_complex_apply.argtypes = [I, S, S, S, S, V, V, V, S, I]
        lib.lfo_qr_complex_solve.argtypes = [I, S, S, S, C.POINTER(C.c_long), C.POINTER(C.c_size_t), V, V, V, V, S, V]
        self.lib = lib

    def elementwise(self, bits, op, a, b=None, c=None, b_index=(1, 0), c_index=(1, 0)):
        out = np.zeros_like(a)
        rc = self.lib.lfo_elementwise(bits, int(op), _ptr(a), _ptr(b), _ptr(c), _ptr(out), a.shape[0],
                                      b_index[0], b_index[1], c_index[0], c_index[1])
        assert rc == 0
        return out

    def mul_chain(self, bits, x, factors):
        """factors: [steps, count, N+3]"""
        out = np.zeros_like(x)
        self.lib.lfo_mul_chain(bits, _ptr(x), _ptr(factors), factors.shape[0], _ptr(out), x.shape[0])
        return out

    def exact_dot_add(self, bits, c, subtract, a, sa, b, sb, K):
        n = bits // 32
        out = np.zeros(n + 3, dtype=np.uint32)
        self.lib.lfo_exact_dot_add_bits(bits, _ptr(c), int(subtract), _ptr(a), sa, _ptr(b), sb, K, _ptr(out))
        return out

    def gemm(self, bits, transpose_a, A, B, m, n, k, C=None, subtract=False, rows=None):
        out = np.zeros((m * n, bits // 32 + 3), dtype=np.uint32) if C is None else C.copy()
        r0, r1 = rows if rows else (0, m)
        self.lib.lfo_gemm_rows(bits, int(transpose_a), _ptr(A), _ptr(B), m, n, k, _ptr(out), int(subtract), r0, r1)
        return out

    def syrk(self, bits, A, rows, cols, C=None, lower_only=True, subtract=False, lines=None):
        out = np.zeros((cols * cols, bits // 32 + 3), dtype=np.uint32) if C is None else C.copy()
        r0, r1 = lines if lines else (0, cols)
        self.lib.lfo_syrk_rows(bits, _ptr(A), rows, cols, _ptr(out), int(lower_only), int(subtract), r0, r1)
        return out

    def cholesky(self, bits, A, n, block=32):
        L = np.zeros_like(A)
        info = (C.c_long * 3)()
        self.lib.lfo_cholesky(bits, _ptr(A), n, _ptr(L), block, info)
        return L, (int(info[0]), int(info[1]), int(info[2]))

    def solve(self, bits, L, n, B, nrhs, block=32, passes=3):
        X = B.copy()
        self.lib.lfo_solve(bits, _ptr(L), n, _ptr(X), nrhs, block, passes)
        return X

    def lu4(self, bits, count, rhs, flags, A, B=None):
        n = bits // 32
        R = 4 if flags & 4 else rhs
        X = np.zeros((count * 4 * R, 2, n + 3), dtype=np.uint32)
        det = np.zeros((count, 2, n + 3), dtype=np.uint32)
        st = np.zeros(count, dtype=np.uint32)
        self.lib.lfo_lu4(bits, count, rhs, flags, _ptr(A), _ptr(B), _ptr(X), _ptr(det), _ptr(st))
        return X, det, st

    def strided_gemm(self, bits, complex_, s, A, B, C):
        out = C.copy()
        self.lib.lfo_strided_gemm(bits, int(complex_), s["count"], s["m"], s["n"], s["k"], s["stride_a"],
                                  s["stride_b"], s["stride_c"], int(s.get("accumulate", False)),
                                  int(s.get("fused", False)), int(s.get("negative", False)),
                                  _ptr(A), _ptr(B), _ptr(out))
        return out

    def cast(self, from_bits, to_bits, complex_, x):
        """x: [count, N+3] or [count, 2, N+3] at from_bits; returns the same shape at to_bits."""
        count = x.shape[0]
        n = to_bits // 32
        out = np.zeros((count, 2, n + 3) if complex_ else (count, n + 3), dtype=np.uint32)
        assert self.lib.lfo_cast(from_bits, to_bits, int(complex_), _ptr(x), _ptr(out), count) == 0
        return out

    def tree_sum(self, bits, complex_, x):
        n = bits // 32
        out = np.zeros((2, n + 3) if complex_ else (n + 3,), dtype=np.uint32)
        src = np.ascontiguousarray(x) if x.shape[0] else np.zeros((1,) + out.shape, dtype=np.uint32)
        assert self.lib.lfo_tree_sum(bits, int(complex_), _ptr(src), x.shape[0], _ptr(out)) == 0
        return out


    def segmented_dot(self, bits, complex_, segments, length, shared, a, b):
        n = bits // 32
        out = np.zeros((segments, 2, n + 3) if complex_ else (segments, n + 3), dtype=np.uint32)
        assert self.lib.lfo_segmented_dot(bits, int(complex_), segments, length, int(shared), _ptr(a), _ptr(b), _ptr(out)) == 0
        return out

    def recurrence(self, bits, seeds, weights, count, steps, states_per_weight=1):
        n = bits // 32
        out = np.zeros((count, 2, n + 3), dtype=np.uint32)
        assert self.lib.lfo_recurrence(bits, _ptr(seeds), _ptr(weights), _ptr(out), count, steps, states_per_weight) == 0
        return out


    def qr(self, bits, A, m, n, block=32, rank_bits=0, pivot=False):
        """Householder QR of A (m x n elements); returns a dict with R, V, T, tau, rank, reason, status,
        recomputed, perm (None unpivoted) and the shape, as the factor the solve and apply calls take."""
        w = bits // 32 + 3
        nb = block if block and block < n else n
        blocks = (n + nb - 1) // nb if nb else 0
        R = np.zeros((n * n, w), dtype=np.uint32)
        V = np.zeros((m * n, w), dtype=np.uint32)
        T = np.zeros((max(blocks * nb * nb, 1), w), dtype=np.uint32)
        tau = np.zeros((max(n, 1), w), dtype=np.uint32)
        info = (C.c_long * 4)()
        A = np.ascontiguousarray(A.reshape(m * n, w)) if m * n else np.zeros((1, w), dtype=np.uint32)
        perm = None
        if pivot:
            pm = (C.c_size_t * max(n, 1))()
            self.lib.lfo_qr_pivoted(bits, _ptr(A), m, n, block, rank_bits, _ptr(R), _ptr(V), _ptr(T), _ptr(tau), pm, info)
            perm = [int(pm[i]) for i in range(n)]
        else:
            self.lib.lfo_qr(bits, _ptr(A), m, n, block, rank_bits, _ptr(R), _ptr(V), _ptr(T), _ptr(tau), info)
        return {"bits": bits, "m": m, "n": n, "block": block, "nb": nb, "R": R, "V": V, "T": T[:blocks * nb * nb],
                "tau": tau[:n], "rank": int(info[0]), "reason": int(info[1]), "status": int(info[2]),
                "recomputed": int(info[3]), "perm": perm}

    def qr_apply(self, f, B, nrhs, transpose):
        """B (m x nrhs) -> Q^T B (transpose) or Q B."""
        out = np.ascontiguousarray(B.copy())
        if f["m"] and nrhs:
            self.lib.lfo_qr_apply(f["bits"], f["m"], f["n"], f["block"], f["rank"], _ptr(f["V"]), _ptr(f["T"]),
                                  _ptr(out), nrhs, int(bool(transpose)))
        return out

    def qr_solve(self, f, B, nrhs):
        """Least-squares X (n x nrhs) from B (m x nrhs)."""
        w = f["bits"] // 32 + 3
        X = np.zeros((max(f["n"] * nrhs, 1), w), dtype=np.uint32)
        info = (C.c_long * 4)(f["rank"], f["reason"], f["status"], f["recomputed"])
        perm = (C.c_size_t * max(f["n"], 1))(*f["perm"]) if f["perm"] is not None else None
        if f["n"] and nrhs:
            self.lib.lfo_qr_solve(f["bits"], f["m"], f["n"], f["block"], info, perm, _ptr(f["R"]), _ptr(f["V"]),
                                  _ptr(f["T"]), _ptr(np.ascontiguousarray(B)), nrhs, _ptr(X))
        return X[:f["n"] * nrhs]


    def exact_gemm4(self, bits, complex_, shape, A, B, C):
        """The exact batched 4 x 4 product; shape: dict(count, stride_a, stride_b, stride_c, accumulate, negative).
        Returns the new C."""
        out = np.ascontiguousarray(C.copy())
        assert self.lib.lfo_exact_gemm4(bits, int(complex_), shape["count"], shape["stride_a"], shape["stride_b"], shape["stride_c"],
                                        int(shape.get("accumulate", False)), int(shape.get("negative", False)),
                                        _ptr(np.ascontiguousarray(A)), _ptr(np.ascontiguousarray(B)), _ptr(out)) == 0
        return out

    def qr_complex(self, bits, A, m, n, block=32, rank_bits=0, pivot=False):
        """Complex Householder QR of A (m * n complex elements, shape [m * n, 2, N + 3]); the factor dict as qr's."""
        w = bits // 32 + 3
        nb = block if block and block < n else n
        blocks = (n + nb - 1) // nb if nb else 0
        R = np.zeros((max(n * n, 1), 2, w), dtype=np.uint32)
        V = np.zeros((max(m * n, 1), 2, w), dtype=np.uint32)
        T = np.zeros((max(blocks * nb * nb, 1), 2, w), dtype=np.uint32)
        tau = np.zeros((max(n, 1), 2, w), dtype=np.uint32)
        info = (C.c_long * 4)()
        pm = (C.c_size_t * max(n, 1))()
        A = np.ascontiguousarray(A.reshape(m * n, 2, w)) if m * n else np.zeros((1, 2, w), dtype=np.uint32)
        self.lib.lfo_qr_complex(bits, _ptr(A), m, n, block, rank_bits, int(bool(pivot)), _ptr(R), _ptr(V), _ptr(T), _ptr(tau), pm, info)
        return {"bits": bits, "m": m, "n": n, "block": block, "nb": nb, "R": R[:n * n], "V": V[:m * n],
                "T": T[:blocks * nb * nb], "tau": tau[:n], "rank": int(info[0]), "reason": int(info[1]),
                "status": int(info[2]), "recomputed": int(info[3]), "perm": [int(pm[i]) for i in range(n)] if pivot else None,
                "complex": True}

    def qr_complex_apply(self, f, B, nrhs, adjoint):
        out = np.ascontiguousarray(B.copy())
        if f["m"] and nrhs:
            self.lib.lfo_qr_complex_apply(f["bits"], f["m"], f["n"], f["block"], f["rank"], _ptr(np.ascontiguousarray(f["V"])),
                                          _ptr(np.ascontiguousarray(f["T"])), _ptr(out), nrhs, int(bool(adjoint)))
        return out

    def qr_complex_solve(self, f, B, nrhs):
        w = f["bits"] // 32 + 3
        X = np.zeros((max(f["n"] * nrhs, 1), 2, w), dtype=np.uint32)
        info = (C.c_long * 4)(f["rank"], f["reason"], f["status"], f["recomputed"])
        perm = (C.c_size_t * max(f["n"], 1))(*f["perm"]) if f["perm"] is not None else None
        if f["n"] and nrhs:
            self.lib.lfo_qr_complex_solve(f["bits"], f["m"], f["n"], f["block"], info, perm, _ptr(np.ascontiguousarray(f["R"])),
                                          _ptr(np.ascontiguousarray(f["V"])), _ptr(np.ascontiguousarray(f["T"])),
                                          _ptr(np.ascontiguousarray(B)), nrhs, _ptr(X))
        return X[:f["n"] * nrhs]


class Reference:
    """The reference's own CPU arithmetic (core.hpp, exact_dot_add) built into oracle/_ref."""

    PATH = os.path.join(HERE, "_ref", "libref.so")

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.PATH)

    def __init__(self) -> None:
        lib = C.CDLL(self.PATH)
        V, S, I, L = C.c_void_p, C.c_size_t, C.c_int, C.c_long
        lib.ref_elementwise.argtypes = [I, I, V, V, V, V, S]
        lib.ref_exact_dot_add.argtypes = [I, V, I, V, L, V, L, S, V]
        lib.ref_dot2_add.argtypes = [I, V, V, V, V, V, V, S]
        lib.ref_divide_word.argtypes = [C.c_uint, C.c_uint, C.c_uint, C.POINTER(C.c_uint), C.POINTER(C.c_uint)]
        lib.ref_qr_blocked.argtypes = [I, V, S, S, S, I, V, V, V, V, C.POINTER(C.c_long)]
        self.lib = lib

    def elementwise(self, bits, op, a, b=None, c=None):
        out = np.zeros_like(a)
        assert self.lib.ref_elementwise(bits, int(op), _ptr(a), _ptr(b), _ptr(c), _ptr(out), a.shape[0]) == 0
        return out

    def exact_dot_add(self, bits, c, subtract, a, sa, b, sb, K):
        out = np.zeros(bits // 32 + 3, dtype=np.uint32)
        self.lib.ref_exact_dot_add(bits, _ptr(c), int(subtract), _ptr(a), sa, _ptr(b), sb, K, _ptr(out))
        return out

    def qr_blocked(self, bits, A, m, n, block=32, rank_bits=0):
        """Unpivoted QR in the library's blocked right-looking form over the reference's own arithmetic."""
        w = bits // 32 + 3
        nb = block if block and block < n else n
        blocks = (n + nb - 1) // nb if nb else 0
        R = np.zeros((max(n * n, 1), w), dtype=np.uint32)
        V = np.zeros((max(m * n, 1), w), dtype=np.uint32)
        T = np.zeros((max(blocks * nb * nb, 1), w), dtype=np.uint32)
        tau = np.zeros((max(n, 1), w), dtype=np.uint32)
        info = (C.c_long * 4)()
        A = np.ascontiguousarray(A.reshape(m * n, w)) if m * n else np.zeros((1, w), dtype=np.uint32)
        self.lib.ref_qr_blocked(bits, _ptr(A), m, n, block, rank_bits, _ptr(R), _ptr(V), _ptr(T), _ptr(tau), info)
        return {"R": R[:n * n], "V": V[:m * n], "T": T[:blocks * nb * nb], "tau": tau[:n], "rank": int(info[0]),
                "reason": int(info[1]), "status": int(info[2])}

    def dot2_add(self, bits, a, b, c, d, e):
        out = np.zeros_like(a)
        self.lib.ref_dot2_add(bits, _ptr(a), _ptr(b), _ptr(c), _ptr(d), _ptr(e), _ptr(out), a.shape[0])
        return out


class Mpfr:
    """Independent MPFR replays (tests/reference.hpp semantics)."""

    def __init__(self) -> None:
        lib = _load("libmpfr_oracle.so")
        V, S, I, L = C.c_void_p, C.c_size_t, C.c_int, C.c_long
        lib.mpo_real.argtypes = [I, I, V, V, V, S]
        lib.mpo_fused.argtypes = [I, I, V, V, V, V, S]
        lib.mpo_dot.argtypes = [I, V, I, V, L, V, L, S, V]
        lib.mpo_dot2_add.argtypes = [I, V, V, V, V, V, V, S]
        lib.mpo_cast.argtypes = [I, I, V, V, S]
        lib.mpo_chain_setup.argtypes = [I, V, V, S, S]
        lib.mpo_chain_setup.restype = V
        lib.mpo_chain_run.argtypes = [V, I]
        lib.mpo_chain_run.restype = C.c_double
        lib.mpo_chain_result.argtypes = [V, V]
        lib.mpo_chain_free.argtypes = [V]
        self.lib = lib

    def chain_baseline(self, bits, x, factors, threads_list, warmup=2, samples=9):
        """The MPFR chain baseline (benchmarks/benchmark.cpp method): median pass seconds for each thread
        count in threads_list (passes of the counts alternate, as the reference alternates serial and
        parallel runs), and the result values of the last pass."""
        h = self.lib.mpo_chain_setup(bits, _ptr(x), _ptr(factors), factors.shape[0], x.shape[0])
        try:
            times = {t: [] for t in threads_list}
            for i in range(warmup + samples):
                for t in threads_list:
                    s = self.lib.mpo_chain_run(h, t)
                    if i >= warmup:
                        times[t].append(s)
            out = np.zeros_like(x)
            self.lib.mpo_chain_result(h, _ptr(out))
        finally:
            self.lib.mpo_chain_free(h)
        return {t: float(np.median(v)) for t, v in times.items()}, out

    def cast(self, from_bits, to_bits, x):
        """Real components x [count, N+3] at from_bits, rounded to to_bits."""
        out = np.zeros((x.shape[0], to_bits // 32 + 3), dtype=np.uint32)
        assert self.lib.mpo_cast(from_bits, to_bits, _ptr(x), _ptr(out), x.shape[0]) == 0
        return out

    def dot(self, bits, c, subtract, a, sa, b, sb, K):
        """RN(c -/+ sum_k a[k sa] b[k sb]) by mpfr_sum (c may be None)."""
        out = np.zeros(bits // 32 + 3, dtype=np.uint32)
        self.lib.mpo_dot(bits, _ptr(c), int(subtract), _ptr(a), sa, _ptr(b), sb, K, _ptr(out))
        return out

    def real(self, bits, op, a, b=None):
        out = np.zeros_like(a)
        assert self.lib.mpo_real(bits, int(op), _ptr(a), _ptr(b), _ptr(out), a.shape[0]) == 0
        return out

    def fused(self, bits, subtract, a, b, c):
        out = np.zeros_like(a)
        self.lib.mpo_fused(bits, int(subtract), _ptr(a), _ptr(b), _ptr(c), _ptr(out), a.shape[0])
        return out

    def dot(self, bits, c, subtract, a, sa, b, sb, K):
        out = np.zeros(bits // 32 + 3, dtype=np.uint32)
        self.lib.mpo_dot(bits, _ptr(c), int(subtract), _ptr(a), sa, _ptr(b), sb, K, _ptr(out))
        return out

    def dot2_add(self, bits, a, b, c, d, e):
        out = np.zeros_like(a)
        self.lib.mpo_dot2_add(bits, _ptr(a), _ptr(b), _ptr(c), _ptr(d), _ptr(e), _ptr(out), a.shape[0])
        return out

    # composed complex replays (tests/reference.hpp:45-55)
    def complex(self, bits, op, a, b):
        re = lambda z: np.ascontiguousarray(z[:, 0])
        im = lambda z: np.ascontiguousarray(z[:, 1])
        R = lambda o, x, y: self.real(bits, o, x, y)
        if op == 4:
            r, i = R(0, re(a), re(b)), R(0, im(a), im(b))
        elif op == 5:
            r = R(1, R(2, re(a), re(b)), R(2, im(a), im(b)))
            i = R(0, R(2, re(a), im(b)), R(2, im(a), re(b)))
        else:
            d = R(0, R(2, re(b), re(b)), R(2, im(b), im(b)))
            r = R(3, R(0, R(2, re(a), re(b)), R(2, im(a), im(b))), d)
            i = R(3, R(1, R(2, im(a), re(b)), R(2, re(a), im(b))), d)
        return np.ascontiguousarray(np.stack([r, i], axis=1))
