"""CPU: the C-ABI library builds, loads and exports every symbol include/*.h declares; the
Python mirror's pure host logic (broadcast counts, operation classes) matches the reference.
No kernel is launched here."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?(?:int|void|size_t|char|unsigned)\s*\*?\s*(lf_\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def library():
    from limbforge_b200 import build
    path = build.build()
    return ctypes.CDLL(path)


def test_header_declares_the_boundary():
    names = declared_symbols()
    for required in ("lf_engine_run", "lf_engine_run_ternary", "lf_batch_submit", "lf_submission_wait",
                     "lf_buffer_mapped", "lf_engine_lu4", "lf_batched_gemm", "lf_dev_mul_chain"):
        assert required in names


def test_library_exports_every_declared_symbol(library):
    missing = [n for n in declared_symbols() if not hasattr(library, n)]
    assert not missing, f"declared in include/*.h but not exported: {missing}"


def test_library_loads_without_a_gpu_and_reports_errors(library):
    library.lf_version.restype = ctypes.c_char_p
    assert b"sm_100a" in library.lf_version()
    library.lf_last_error.restype = ctypes.c_char_p
    # invalid width is rejected on the host before any device work
    rc = library.lf_dev_elementwise(100, 2, None, None, None, None, ctypes.c_size_t(4),
                                    (ctypes.c_size_t * 2)(1, 0), (ctypes.c_size_t * 2)(1, 0), None)
    assert rc == 1
    assert b"multiple of 32" in library.lf_last_error()


def test_broadcast_and_operation_classes():
    from limbforge_b200.api import (Broadcast, InvalidArgument, LogicError, Operation, broadcast_elements,
                                    operation_is_complex, operation_is_ternary, operation_is_unary)
    assert broadcast_elements(1001, Broadcast(4, 0)) == 251
    assert broadcast_elements(1001, Broadcast(1, 7)) == 7
    assert broadcast_elements(1001, Broadcast(3, 5)) == 5
    assert broadcast_elements(1001, Broadcast(1001, 0)) == 1
    with pytest.raises(InvalidArgument):
        broadcast_elements(4, Broadcast(0, 0))
    assert issubclass(InvalidArgument, LogicError)
    assert [operation_is_complex(o) for o in Operation] == [False] * 4 + [True] * 3 + [False] * 4 + [True] * 2
    assert [o for o in Operation if operation_is_unary(o)] == [Operation.square, Operation.sqrt]
    assert [o for o in Operation if operation_is_ternary(o)] == [Operation.fma, Operation.fms, Operation.complex_fma,
                                                                  Operation.complex_fms]
