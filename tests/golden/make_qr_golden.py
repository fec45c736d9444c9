"""Generates tests/golden/qr_golden.npz (run from the repository root with the reference checkout present:
``python tests/golden/make_qr_golden.py``).

Inputs are fixture classes of the reference's tests/test_qr.cpp (tests/qr_cases.py regenerates them with numpy
seeds).  Expected factors come from oracle/_ref/libref.so's ``ref_qr_blocked``: the library's blocked
right-looking Householder sequence evaluated with the reference's own exact_dot / exact_dot_add / sqrt / sub /
div / mul compiled from its sources.  Generation fails unless the C oracle's column-by-column statement
(lf_oracle.c) gives the same bits.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle.oracle import Oracle, Reference  # noqa: E402
from tests import qr_cases as qc  # noqa: E402

CASES = [  # bits, m, n, kind, block, rank_bits
    (256, 33, 7, "moderate", 32, 0),
    (256, 48, 24, "qsc", 16, 0),
    (256, 40, 21, "graded", 7, 0),
    (64, 40, 20, "spread", 7, 0),
    (384, 20, 12, "wide", 5, 0),
    (224, 41, 7, "dependent", 16, 112),
]


def main() -> None:
    ref, orc = Reference(), Oracle()
    rng = np.random.default_rng(4321)
    out = {}
    cases = []
    for bits, m, n, kind, block, rank_bits in CASES:
        cases.append((f"{kind}_{bits}_{m}x{n}", bits, qc.matrix(bits, m, n, kind, rng), m, n, block, rank_bits))
    for label, A, m, n, rank_bits, _ in qc.special_cases(256, rng):
        cases.append((label.replace(" ", "_").replace(",", "").replace("(", "").replace(")", ""), 256, A, m, n, 8, rank_bits))
    for i, (label, bits, A, m, n, block, rank_bits) in enumerate(cases):
        want = ref.qr_blocked(bits, A, m, n, block, rank_bits)
        got = orc.qr(bits, A, m, n, block, rank_bits)
        for k in ("R", "V", "T", "tau"):
            assert (got[k] == want[k]).all(), f"{label}: oracle {k} differs from the reference build"
        assert (got["rank"], got["reason"], got["status"]) == (want["rank"], want["reason"], want["status"]), label
        key = f"c{i}"
        out[f"{key}_A"] = A
        out[f"{key}_meta"] = np.array([bits, m, n, block, rank_bits, want["rank"], want["reason"], want["status"]], dtype=np.int64)
        for k in ("R", "V", "T", "tau"):
            out[f"{key}_{k}"] = want[k]
        out[f"{key}_label"] = np.array(label)
    out["count"] = np.array(len(cases))
    path = os.path.join(ROOT, "tests", "golden", "qr_golden.npz")
    np.savez_compressed(path, **out)
    print(f"{len(cases)} QR cases -> {path} ({os.path.getsize(path)} bytes)")


if __name__ == "__main__":
    main()
