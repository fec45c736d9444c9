"""CPU: the scalar host arithmetic of the C++17 drop-in headers (include/limbforge/core.hpp: add, sub, mul, div,
square, sqrt, fma, fms, dot2_add and the complex forms; linalg.hpp: exact_dot_add / exact_dot), compiled with g++
alone from the same source as the GPU kernels, against the C oracle bit for bit at four widths.  Inputs include
exact zeros, sparse significands (exact results and ties), wide exponent gaps and cancellation."""
import os
import subprocess

import numpy as np
import pytest

from fused_cases import dot2_cases
from limbforge_b200 import numbers as nb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("host") / "host_arith")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", f"-I{os.path.join(ROOT, 'include')}",
                    os.path.join(ROOT, "tests", "cpp", "host_arith.cpp"), "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("bits", [64, 256, 416, 1024])
def test_host_scalar_arithmetic_vs_oracle(program, oracle, tmp_path, bits):
    rng = np.random.default_rng(bits + 1)
    n = bits // 32
    cnt = 96
    ops = [nb.random_numbers(rng, cnt, bits, 300, zero_frac=0.05, sparse_frac=0.1) for _ in range(5)]
    a, b, c, d, e = ops
    b[::4, n] = (nb.exponent(a[::4]) - rng.integers(0, bits + 80, size=a[::4].shape[0])).astype(np.int32).view(np.uint32)
    b[1::9] = nb.negate(a[1::9])
    fa, fb, fc = dot2_cases(rng, bits, cnt)                # adversarial three-term sums in the complex fma slots
    c[::2], d[::2], e[::2] = fb[::2, 0], fb[::2, 1], fc[::2, 0]
    a[::2], b[::2] = fa[::2, 0], fa[::2, 1]
    src = tmp_path / "in.bin"
    with open(src, "wb") as fh:
        fh.write(np.uint64(cnt).tobytes())
        for x in (a, b, c, d, e):
            fh.write(np.ascontiguousarray(x).tobytes())
    dst = tmp_path / "out.bin"
    subprocess.run([program, str(bits), str(src), str(dst)], check=True)
    got = np.fromfile(dst, dtype=np.uint32).reshape(-1, n + 3)
    per = 9 + 10
    rows = got[:cnt * per].reshape(cnt, per, n + 3)
    E = lambda op, *xs: oracle.elementwise(bits, op, *[np.ascontiguousarray(x) for x in xs])
    r = a.copy()
    r[:, n + 1] = np.abs(nb.sign(r)).astype(np.int32).view(np.uint32)
    want = [E(0, a, b), E(1, a, b), E(2, a, b), E(3, a, b), E(7, a), E(8, r), E(9, a, b, c), E(10, a, b, c)]
    want.append(np.stack([_dot2(oracle, bits, a[i], b[i], c[i], d[i], e[i]) for i in range(cnt)]))
    x = np.stack([a, b], axis=1); y = np.stack([c, d], axis=1); z = np.stack([e, a], axis=1)
    for op in (4, 5, 6, 11, 12):
        w = E(op, x, y, z) if op in (11, 12) else E(op, x, y)
        want += [w[:, 0], w[:, 1]]
    for k, w in enumerate(want):
        assert (rows[:, k] == w).all(), f"bits={bits} result {k} differs at {np.nonzero((rows[:, k] != w).any(axis=1))[0][:5]}"
    assert (got[cnt * per] == oracle.exact_dot_add(bits, c[0], 1, a, 1, b, 1, cnt)).all(), "exact_dot_add"
    assert (got[cnt * per + 1] == oracle.exact_dot_add(bits, None, 0, a, 1, d, 1, cnt)).all(), "exact_dot"


def _dot2(oracle, bits, a, b, c, d, e):
    import ctypes as C
    out = np.zeros_like(a)
    p = lambda v: np.ascontiguousarray(v).ctypes.data_as(C.c_void_p)
    oracle.lib.lfo_dot2_add(bits // 32, p(a), p(b), p(c), p(d), p(e), out.ctypes.data_as(C.c_void_p))
    return out


def test_wide_clusters_stream_exactly(tmp_path):
    """Exact sums whose clusters are wider than the accumulator window (tests/cpp/wide_sum.cpp): the streaming path of
    cluster_round with the smallest window (8N + 4 words) gives the same bits as a window wide enough for every cluster,
    at six widths, over chains of products spaced below the cluster gap, exact cancellations, ties and far terms."""
    exe = str(tmp_path / "wide_sum")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", f"-I{os.path.join(ROOT, 'include')}",
                    os.path.join(ROOT, "tests", "cpp", "wide_sum.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "mismatches 0" in r.stdout, r.stdout + r.stderr
