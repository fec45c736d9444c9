"""CPU: the MPFR/MPC bridge (include/limbforge/mpfr_bridge.hpp, the reference's mpfr_bridge.hpp) compiled with g++
against the installed MPFR/GMP runtime libraries.  from_mpfr of exact 1024-bit values at five widths and to_mpfr at
those precisions must equal the oracle's precision cast (itself pinned to mpfr_set); precisions that are not whole
words must equal MPFR's own rounding; the program's self checks cover specials, the exponent limits, carries, ties,
the inexact flag, MPFR's range rule, threaded and runtime-width arrays, statuses, decimals and the mpc_t forms."""
import os
import subprocess

import numpy as np
import pytest

from limbforge_b200 import numbers as nb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WIDTHS = [64, 96, 256, 736, 1024]


@pytest.fixture(scope="module")
def bridge(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("bridge") / "bridge")
    # this image has the MPFR/GMP runtime libraries but no headers: tests/cpp/mpfr_decl declares what the bridge uses
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{ROOT}/include", f"-I{ROOT}/tests/cpp/mpfr_decl",
                    os.path.join(ROOT, "tests", "cpp", "bridge.cpp"), "-o", exe, "-l:libmpfr.so.6", "-l:libgmp.so.10",
                    "-pthread"], check=True)
    return exe


def test_bridge_self_checks(bridge):
    r = subprocess.run([bridge, "self"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "bridge ok" in r.stdout, r.stdout + r.stderr


def test_bridge_vs_oracle_cast(bridge, oracle, tmp_path):
    rng = np.random.default_rng(12)
    x = nb.random_numbers(rng, 3000, 1024, 3000, zero_frac=0.02, sparse_frac=0.2)
    x[:64, :32] = 0xFFFFFFFF                                  # all-ones significands: rounding carries at every width
    x[64:128, :31] = 0
    x[64:128, 31] = 0x80000000
    x[64:128, 10] = 0x80000000                                # exact ties at several widths
    x[:128, 33] = np.where(x[:128, 33] == 0, 1, x[:128, 33])  # those rows are nonzero values
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    np.ascontiguousarray(x).tofile(src)
    r = subprocess.run([bridge, "check", str(src), str(len(x)), str(dst)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = np.fromfile(dst, dtype=np.uint32)
    per = sum(w // 32 + 3 + 35 for w in WIDTHS)
    raw = raw.reshape(len(x), per)
    o = 0
    for w in WIDTHS:
        n = w // 32 + 3
        got_from = raw[:, o:o + n]
        got_to = raw[:, o + n:o + n + 35]
        o += n + 35
        narrow = oracle.cast(1024, w, False, x)
        assert (got_from == narrow).all(), f"from_mpfr<{w}>"
        assert (got_to == oracle.cast(w, 1024, False, narrow)).all(), f"to_mpfr at precision {w}"


@pytest.mark.gpu
def test_bridge_buffers_and_inline_import_on_gpu(tmp_path):
    """The engine-buffer forms of the bridge and the inline MPC import, through the C++ headers and the library."""
    from limbforge_b200 import build
    build.build()
    exe = str(tmp_path / "bridge_gpu")
    libdir = os.path.join(ROOT, "limbforge_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{ROOT}/include", f"-I{ROOT}/tests/cpp/mpfr_decl",
                    os.path.join(ROOT, "tests", "cpp", "bridge_gpu.cpp"), "-o", exe, f"-L{libdir}", "-llimbforge_b200",
                    f"-Wl,-rpath,{libdir}", "-l:libmpfr.so.6", "-l:libgmp.so.10", "-pthread"], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "bridge gpu ok" in r.stdout, r.stdout + r.stderr
