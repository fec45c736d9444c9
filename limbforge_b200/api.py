"""Python mirror of the limbforge C++ API over the C ABI (include/limbforge_b200.h).

Names, argument meaning and error classes follow the reference's headers
(include/limbforge/engine.hpp, batched_linalg.hpp, linalg.hpp): ``Engine.run/run_unary/
run_ternary/lu4/make_buffer/batch``, ``Buffer.size/mapped/upload/download``,
``CommandBatch.run/lu4/submit``, ``Submission.ready/wait``, ``BatchedLinalg.gemm`` and
``Linalg.gemm/syrk/cholesky/trsm/cholesky_solve``.  Elements are numpy ``uint32`` arrays in
the reference's struct layout (see ``limbforge_b200.numbers``).  Errors raise
``InvalidArgument`` (std::invalid_argument), ``LogicError`` (std::logic_error) and
``RuntimeFailure`` (std::runtime_error).  Every call goes to the CUDA library; there is no
CPU fallback: a missing or unloadable library raises at import.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
from dataclasses import dataclass

import numpy as np

from .numbers import check_bits, element_words

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "liblimbforge_b200.so")


class LogicError(Exception):
    """std::logic_error"""


class InvalidArgument(LogicError, ValueError):
    """std::invalid_argument"""


class RuntimeFailure(RuntimeError):
    """std::runtime_error"""


class Operation(enum.IntEnum):                                   # engine.hpp:13
    add = 0
    sub = 1
    mul = 2
    div = 3
    complex_add = 4
    complex_mul = 5
    complex_div = 6
    square = 7
    sqrt = 8
    fma = 9
    fms = 10
    complex_fma = 11
    complex_fms = 12


def operation_is_complex(op) -> bool:
    op = int(op)
    return 4 <= op <= 6 or op in (11, 12)


def operation_is_unary(op) -> bool:
    return int(op) in (7, 8)


def operation_is_ternary(op) -> bool:
    return 9 <= int(op) <= 12


@dataclass
class Broadcast:                                                 # engine.hpp:21
    stride: int = 1
    period: int = 0


def broadcast_elements(count: int, b: Broadcast) -> int:         # engine.hpp:22-25
    if not b.stride:
        raise InvalidArgument("broadcast stride must be positive")
    n = count // b.stride + (count % b.stride != 0)
    return b.period if b.period and b.period < n else n


@dataclass
class Timing:                                                    # engine.hpp:18
    gpu_seconds: float = 0.0
    wall_seconds: float = 0.0


@dataclass
class Batched4:                                                  # engine.hpp:36
    count: int = 0
    rhs: int = 0
    inverse: bool = False
    determinant: bool = False
    fused: bool = False


@dataclass
class SegmentedDot:                                              # engine.hpp:30-32
    segments: int = 0
    length: int = 0
    shared_right: bool = False


@dataclass
class ExactGemm4Shape:                                           # experiments/exact_gemm4/prototype.hpp:6
    count: int = 1
    stride_a: int = 16
    stride_b: int = 16
    stride_c: int = 16
    accumulate: bool = False
    negative: bool = False


@dataclass
class ExactGemm4Report:                                          # experiments/exact_gemm4/prototype.hpp:7
    gpu_components: int = 0
    host_components: int = 0
    provisional_reads: bool = False


@dataclass
class StridedGemm:                                               # batched_linalg.hpp:11-14
    count: int = 1
    m: int = 0
    n: int = 0
    k: int = 0
    stride_a: int = 0
    stride_b: int = 0
    stride_c: int = 0
    accumulate: bool = False
    fused: bool = False
    negative: bool = False


@dataclass
class LinalgOptions:                                             # linalg.hpp:18-25
    band_bits: int = 64
    max_bands: int = 4
    max_spread: int = 512
    host_threads: int = 0
    force_fallback: bool = False
    resident_bands: int = 2
    method: int = 0          # 0 auto (residue engine where it applies), 1 generic limb kernel, 2 residue only


@dataclass
class FactorOptions:                                             # linalg.hpp:73-78
    block: int = 32
    host_macs: float = 5e4
    solve_host_macs: float = 4e5
    gpu: bool = True


@dataclass
class CholeskyInfo:                                              # linalg.hpp:82-87
    pivot: int = 0
    pivot_sign: int = 0
    pivot_status: int = 0
    timing: "Timing" = None
    blocks: int = 0
    gpu_updates: int = 0
    host_updates: int = 0
    panel_seconds: float = 0.0
    update_seconds: float = 0.0


@dataclass
class QROptions(FactorOptions):                                  # linalg.hpp:94
    rank_bits: int = 0
    pivot: bool = False


@dataclass
class QRInfo:                                                    # linalg.hpp:98-105
    rank: int = 0
    reason: int = 0          # 0 full rank, 1 zero column, 2 small column, 3 status column
    status: int = 0
    timing: "Timing" = None
    blocks: int = 0
    gpu_updates: int = 0
    host_updates: int = 0
    panel_seconds: float = 0.0
    update_seconds: float = 0.0
    norm_recomputations: int = 0


class _Timing(C.Structure):
    _fields_ = [("gpu_seconds", C.c_double), ("wall_seconds", C.c_double)]


class _Broadcast(C.Structure):
    _fields_ = [("stride", C.c_size_t), ("period", C.c_size_t)]


class _EngineOptions(C.Structure):
    _fields_ = [("threads_per_threadgroup", C.c_uint), ("cooperative_reductions", C.c_int),
                ("cooperative_recurrence", C.c_int), ("device", C.c_int)]


class _Batched4(C.Structure):
    _fields_ = [("count", C.c_size_t), ("rhs", C.c_uint), ("inverse", C.c_int), ("determinant", C.c_int), ("fused", C.c_int)]


class _SegmentedDot(C.Structure):
    _fields_ = [("segments", C.c_size_t), ("length", C.c_size_t), ("shared_right", C.c_int)]


class _ExactGemm4Shape(C.Structure):
    _fields_ = [(f, C.c_size_t) for f in ("count", "stride_a", "stride_b", "stride_c")] + \
               [("accumulate", C.c_int), ("negative", C.c_int)]


class _ExactGemm4Report(C.Structure):
    _fields_ = [("gpu_components", C.c_size_t), ("host_components", C.c_size_t), ("provisional_reads", C.c_int)]


class _StridedGemm(C.Structure):
    _fields_ = [("count", C.c_size_t), ("m", C.c_size_t), ("n", C.c_size_t), ("k", C.c_size_t),
                ("stride_a", C.c_size_t), ("stride_b", C.c_size_t), ("stride_c", C.c_size_t),
                ("accumulate", C.c_int), ("fused", C.c_int), ("negative", C.c_int)]


class _LinalgOptions(C.Structure):
    _fields_ = [("band_bits", C.c_int), ("max_bands", C.c_int), ("max_spread", C.c_int), ("host_threads", C.c_uint),
                ("force_fallback", C.c_int), ("resident_bands", C.c_int), ("method", C.c_int)]


class _FactorOptions(C.Structure):
    _fields_ = [("block", C.c_size_t), ("host_macs", C.c_double), ("solve_host_macs", C.c_double), ("gpu", C.c_int)]


class _CholeskyInfo(C.Structure):
    _fields_ = [("pivot", C.c_size_t), ("pivot_sign", C.c_int), ("pivot_status", C.c_uint32), ("timing", _Timing),
                ("blocks", C.c_size_t), ("gpu_updates", C.c_size_t), ("host_updates", C.c_size_t),
                ("panel_seconds", C.c_double), ("update_seconds", C.c_double)]


class _QROptions(C.Structure):
    _fields_ = [("block", C.c_size_t), ("host_macs", C.c_double), ("solve_host_macs", C.c_double), ("gpu", C.c_int),
                ("rank_bits", C.c_int), ("pivot", C.c_int)]


class _QRInfo(C.Structure):
    _fields_ = [("rank", C.c_size_t), ("reason", C.c_int), ("status", C.c_uint32), ("timing", _Timing),
                ("blocks", C.c_size_t), ("gpu_updates", C.c_size_t), ("host_updates", C.c_size_t),
                ("panel_seconds", C.c_double), ("update_seconds", C.c_double), ("norm_recomputations", C.c_size_t)]


class _LinalgWorkspaces(C.Structure):
    _fields_ = [(f, C.c_size_t) for f in ("scratch_bytes", "idle_bytes", "busy_bytes", "busy_workspaces")]


class _LinalgReport(C.Structure):
    _fields_ = [(f, C.c_size_t) for f in ("m", "n", "k", "gpu_outputs", "trivial_outputs", "gemm_rows", "gemm_cols",
                                          "int8_gemms", "moduli", "band_bits")] + \
               [("analysis_seconds", C.c_double), ("gpu_seconds", C.c_double), ("method", C.c_int)] + \
               [(f, C.c_size_t) for f in ("left_lines", "left_zero_lines", "right_lines", "right_zero_lines")]


class _RaggedLu4(C.Structure):
    _fields_ = [("bits", C.c_int), ("shape", _Batched4), ("A", C.c_uint64), ("B", C.c_uint64), ("X", C.c_uint64),
                ("det", C.c_uint64), ("status", C.c_uint64)]


class _RaggedClassInfo(C.Structure):
    _fields_ = [("bits", C.c_int), ("items", C.c_size_t), ("cells", C.c_size_t), ("block", C.c_uint), ("grid", C.c_uint),
                ("trial_ms", C.c_double)]


class _RaggedInfo(C.Structure):
    _fields_ = [("classes", C.c_size_t), ("cls", _RaggedClassInfo * 31), ("lu4_block", C.c_uint), ("lu4_grid", C.c_uint),
                ("lu4_trial_ms", C.c_double), ("tuned", C.c_int)]


# lf_inline_complex_record (BatchedLinalg::import_inline_complex) as a numpy record.
INLINE_RECORD_DTYPE = np.dtype({"names": ["real_offset", "imag_offset", "real_exponent", "imag_exponent", "real_sign", "imag_sign",
                                          "real_status", "imag_status"],
                                "formats": [np.uint64, np.uint64, np.int32, np.int32, np.int32, np.int32, np.uint32, np.uint32],
                                "offsets": [0, 8, 16, 20, 24, 28, 32, 36], "itemsize": 40})


def page_aligned(nbytes: int) -> np.ndarray:
    """A zeroed uint8 array of whole pages at a page boundary (an anonymous mapping), as inline staging requires."""
    import mmap
    page = mmap.PAGESIZE
    size = max(page, (nbytes + page - 1) // page * page)
    return np.frombuffer(mmap.mmap(-1, size), dtype=np.uint8)


# lf_ragged_gemm as a numpy record (one row per instance); offsets a, b, c are bytes in the arena.
RAGGED_DTYPE = np.dtype({"names": ["bits", "m", "n", "k", "a", "b", "c", "accumulate", "negative"],
                         "formats": [np.int32, np.uint32, np.uint32, np.uint32, np.uint64, np.uint64, np.uint64, np.int32, np.int32],
                         "offsets": [0, 4, 8, 12, 16, 24, 32, 40, 44], "itemsize": 48})


def _load() -> C.CDLL:
    if not os.path.exists(LIBRARY):
        raise ImportError(f"{LIBRARY} is missing: run limbforge_b200.build.build() (nvcc, sm_100a)")
    lib = C.CDLL(LIBRARY)
    P, V, S, I = C.POINTER, C.c_void_p, C.c_size_t, C.c_int
    sig = {
        "lf_last_error": ([], C.c_char_p), "lf_version": ([], C.c_char_p),
        "lf_engine_create": ([P(_EngineOptions), P(V)], I), "lf_engine_destroy": ([V], None),
        "lf_engine_device_name": ([V, C.c_char_p, S], I),
        "lf_engine_run": ([V, I, I, V, V, V, S, _Broadcast, P(_Timing)], I),
        "lf_engine_run_unary": ([V, I, I, V, V, S, P(_Timing)], I),
        "lf_engine_run_ternary": ([V, I, I, V, V, V, V, S, _Broadcast, _Broadcast, P(_Timing)], I),
        "lf_engine_lu4": ([V, I, P(_Batched4), V, V, V, V, V, P(_Timing)], I),
        "lf_batched_gemm": ([V, I, I, P(_StridedGemm), V, V, V, P(_Timing)], I),
        "lf_buffer_create": ([V, S, P(V)], I), "lf_buffer_release": ([V], None), "lf_buffer_bytes": ([V], S),
        "lf_buffer_upload": ([V, V, S], I), "lf_buffer_download": ([V, V, S], I),
        "lf_buffer_mapped": ([V, P(V)], I), "lf_buffer_device_pointer": ([V, P(V)], I),
        "lf_batch_create": ([V, P(V)], I), "lf_batch_destroy": ([V], None),
        "lf_batch_run": ([V, I, I, I, V, V, V, V, S, _Broadcast, _Broadcast], I),
        "lf_batch_lu4": ([V, I, P(_Batched4), V, V, V, V, V], I),
        "lf_batch_strided_gemm": ([V, I, I, P(_StridedGemm), V, V, V], I),
        "lf_batch_submit": ([V, P(V)], I), "lf_submission_ready": ([V, P(I)], I),
        "lf_submission_wait": ([V, P(_Timing)], I), "lf_submission_destroy": ([V], None),
        "lf_dev_elementwise": ([I, I, V, V, V, V, S, _Broadcast, _Broadcast, V], I),
        "lf_host_alloc": ([S, P(V)], I), "lf_host_free": ([V], None),
        "lf_dev_mul_chain": ([I, V, V, S, C.c_uint, V, S, V], I),
        "lf_dev_mul_chain_lanes": ([I, I, V, V, S, C.c_uint, V, S, V], I),
        "lf_linalg_create": ([V, P(_LinalgOptions), P(V)], I), "lf_linalg_destroy": ([V], None),
        "lf_linalg_get_report": ([V, P(_LinalgReport)], I),
        "lf_linalg_gemm": ([V, I, I, V, V, S, S, S, V, I, P(_Timing)], I),
        "lf_linalg_syrk": ([V, I, V, S, S, V, I, I, P(_Timing)], I),
        "lf_linalg_cholesky": ([V, I, V, S, V, P(_FactorOptions), P(_CholeskyInfo)], I),
        "lf_linalg_trsm": ([V, I, I, V, S, V, S, V, P(_FactorOptions), P(_Timing)], I),
        "lf_linalg_cholesky_solve": ([V, I, V, S, V, S, V, P(_FactorOptions), P(_Timing)], I),
        "lf_dev_exact_product": ([V, I, V, S, S, V, S, S, S, S, S, V, S, I, I, V], I),
        "lf_linalg_batch_gemm": ([V, V, I, I, V, V, S, S, S, V, I, P(V)], I),
        "lf_linalg_batch_syrk": ([V, V, I, V, S, S, V, I, I, P(V)], I),
        "lf_linalg_ticket_resolved": ([V, P(I)], I), "lf_linalg_ticket_report": ([V, P(_LinalgReport)], I),
        "lf_linalg_ticket_destroy": ([V], None),
        "lf_linalg_get_workspaces": ([V, P(_LinalgWorkspaces)], I), "lf_linalg_release_workspaces": ([V, P(_LinalgWorkspaces)], I),
        "lf_buffer_holders": ([V], I),
        "lf_engine_cast": ([V, I, I, I, V, V, S, P(_Timing)], I),
        "lf_batch_cast": ([V, I, I, I, V, V, S], I), "lf_batch_tree_sum": ([V, I, I, V, V, S], I),
        "lf_dev_cast": ([I, I, I, V, V, S, V], I), "lf_dev_tree_sum": ([I, I, V, S, V, V, V], I),
        "lf_ragged_pack": ([I, V, S, P(_RaggedLu4), P(C.c_uint64)], I),
        "lf_ragged_plan_create": ([V, I, I, V, S, P(_RaggedLu4), C.c_uint64, P(V)], I),
        "lf_ragged_plan_tune": ([V, V], I), "lf_ragged_plan_run": ([V, V, V], I),
        "lf_ragged_plan_get_info": ([V, P(_RaggedInfo)], I), "lf_ragged_plan_destroy": ([V], None),
        "lf_probe_word_mac_rate": ([I, P(C.c_double)], I),
        "lf_test_residue_wait_limit": ([C.c_uint, P(C.c_uint32)], I),
        "lf_engine_segmented_dot": ([V, I, I, P(_SegmentedDot), V, V, V, P(_Timing)], I),
        "lf_batch_segmented_dot": ([V, I, I, P(_SegmentedDot), V, V, V], I),
        "lf_engine_exact_gemm4": ([V, I, I, P(_ExactGemm4Shape), V, V, V, P(_ExactGemm4Report), P(_Timing)], I),
        "lf_batch_exact_gemm4": ([V, I, I, P(_ExactGemm4Shape), V, V, V], I),
        "lf_batch_import_inline_complex": ([V, I, V, S, V, S, V], I),
        "lf_engine_recurrence": ([V, I, V, V, V, S, C.c_uint, C.c_uint, P(_Timing)], I),
        "lf_linalg_factor_qr": ([V, I, V, S, S, P(_QROptions), P(V)], I),
        "lf_linalg_factor_qr_augmented": ([V, I, V, S, S, V, P(_QROptions), P(V)], I),
        "lf_linalg_factor_qr_buffer": ([V, I, V, S, S, P(_QROptions), P(V)], I),
        "lf_qr_destroy": ([V], None),
        "lf_qr_describe": ([V, P(I), P(S), P(S), P(S), P(I), P(_QRInfo)], I),
        "lf_qr_r": ([V], V), "lf_qr_v": ([V], V), "lf_qr_tau": ([V], V), "lf_qr_t": ([V], V),
        "lf_qr_permutation": ([V], P(S)),
        "lf_qr_solve": ([V, V, S, V, P(_Timing)], I), "lf_qr_apply_q": ([V, V, S, I, P(_Timing)], I),
        "lf_qr_solve_buffers": ([V, V, S, V, P(_Timing)], I), "lf_qr_apply_q_buffer": ([V, V, S, I, P(_Timing)], I),
        "lf_linalg_factor_qr_complex": ([V, I, V, S, S, P(_QROptions), P(V)], I), "lf_qr_is_complex": ([V], I),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes, f.restype = args, res
    return lib


lib = _load()


def check(rc: int) -> None:
    if rc == 0:
        return
    msg = lib.lf_last_error().decode()
    if rc == 1:
        raise InvalidArgument(msg)
    if rc == 2:
        raise LogicError(msg)
    raise RuntimeFailure(msg)


def _ptr(a) -> C.c_void_p | None:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise InvalidArgument("arrays must be C contiguous")
        return C.c_void_p(a.ctypes.data)
    return C.c_void_p(int(a))


def _bc(b: Broadcast | None) -> _Broadcast:
    b = b or Broadcast()
    return _Broadcast(b.stride, b.period)


def _timing(t: _Timing) -> Timing:
    return Timing(t.gpu_seconds, t.wall_seconds)


def _elements(a: np.ndarray) -> int:
    return a.shape[0] if a.ndim >= 1 else 0


class Buffer:
    """Device-resident typed storage (engine.hpp:74-86).  ``bits=0`` holds uint32 words."""

    def __init__(self, engine: "Engine", count: int, bits: int, complex_: bool):
        self.engine, self.count, self.bits, self.complex = engine, count, bits, complex_
        self.words = (element_words(bits) * (2 if complex_ else 1)) if bits else 1
        h = C.c_void_p()
        check(lib.lf_buffer_create(engine.handle, 4 * self.words * count, C.byref(h)))
        self.handle = h

    def __del__(self):
        if getattr(self, "handle", None) and lib is not None:
            lib.lf_buffer_release(self.handle)
            self.handle = None

    def size(self) -> int:
        return self.count

    def _shape(self, n):
        if not self.bits:
            return (n,)
        return (n, 2, self.words // 2) if self.complex else (n, self.words)

    def upload(self, source: np.ndarray, count: int | None = None) -> None:
        n = _elements(source) if count is None else count
        if n > self.count:
            raise InvalidArgument("upload exceeds buffer")
        src = np.ascontiguousarray(source, dtype=np.uint32)
        check(lib.lf_buffer_upload(self.handle, _ptr(src), 4 * self.words * n))

    def download(self, count: int | None = None, out: np.ndarray | None = None) -> np.ndarray:
        n = self.count if count is None else count
        if n > self.count:
            raise InvalidArgument("download exceeds buffer")
        dst = np.empty(self._shape(n), dtype=np.uint32) if out is None else out
        check(lib.lf_buffer_download(self.handle, _ptr(dst), 4 * self.words * n))
        return dst

    def mapped(self) -> np.ndarray:
        """Host view (engine.hpp:82); writes reach the device at the next submission using it."""
        p = C.c_void_p()
        check(lib.lf_buffer_mapped(self.handle, C.byref(p)))
        n = self.count * self.words
        arr = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint32)), shape=(max(n, 1),))[:n]
        return arr.reshape(self._shape(self.count))

    def device_pointer(self) -> int:
        p = C.c_void_p()
        check(lib.lf_buffer_device_pointer(self.handle, C.byref(p)))
        return p.value or 0


class Submission:
    def __init__(self, handle, completions=()):
        self.handle = handle
        self._completions = list(completions)

    def __del__(self):
        if getattr(self, "handle", None) and lib is not None:
            lib.lf_submission_destroy(self.handle)
            self.handle = None

    def ready(self) -> bool:
        r = C.c_int()
        check(lib.lf_submission_ready(self.handle, C.byref(r)))
        return bool(r.value)

    def wait(self) -> Timing:
        t = _Timing()
        check(lib.lf_submission_wait(self.handle, C.byref(t)))
        for f in self._completions:
            f()
        self._completions = []
        return _timing(t)


class CommandBatch:
    """Asynchronous batch of resident operations (engine.hpp:104-182)."""

    def __init__(self, engine: "Engine"):
        self.engine = engine
        h = C.c_void_p()
        check(lib.lf_batch_create(engine.handle, C.byref(h)))
        self.handle = h
        self._completions = []      # run once the submission has been waited for (tickets)

    def __del__(self):
        if getattr(self, "handle", None) and lib is not None:
            lib.lf_batch_destroy(self.handle)
            self.handle = None

    def run(self, op, a: Buffer, b: Buffer | None = None, c: Buffer | None = None, out: Buffer | None = None,
            b_index: Broadcast | None = None, c_index: Broadcast | None = None) -> None:
        """run(op, a, b, out[, b_index]) / run(op, a, b, c, out[, b_index, c_index]) / run(op, a, out)"""
        op = Operation(op)
        if operation_is_unary(op):
            out = out if out is not None else b
            b = None
        elif not operation_is_ternary(op):
            out = out if out is not None else c
            c = None
        if out is None:
            raise InvalidArgument("operation requires a different number of inputs")
        if b_index is None and c_index is None:
            same = [x for x in (a, b, c, out) if x is not None]
            if any(x.count != a.count for x in same):
                raise InvalidArgument("buffer counts must match")
        elif a.count != out.count:
            raise InvalidArgument("buffer counts do not match the broadcast")
        check(lib.lf_batch_run(self.handle, a.bits, int(a.complex), int(op), a.handle, b.handle if b else None,
                               c.handle if c else None, out.handle, a.count, _bc(b_index), _bc(c_index)))

    def lu4(self, shape: Batched4, A: Buffer, B: Buffer | None, X: Buffer, det: Buffer | None, status: Buffer) -> None:
        s = _Batched4(shape.count, shape.rhs, int(shape.inverse), int(shape.determinant), int(shape.fused))
        check(lib.lf_batch_lu4(self.handle, A.bits, C.byref(s), A.handle, B.handle if B else None, X.handle if X else None,
                               det.handle if det else None, status.handle))

    def segmented_dot(self, shape: SegmentedDot, a: Buffer, b: Buffer, out: Buffer) -> None:
        """CommandBatch::segmented_dot (engine.hpp:174)."""
        sh = _SegmentedDot(shape.segments, shape.length, int(shape.shared_right))
        check(lib.lf_batch_segmented_dot(self.handle, a.bits, int(a.complex), C.byref(sh), a.handle, b.handle, out.handle))

    def cast(self, a: Buffer, out: Buffer) -> None:
        """CommandBatch::cast (engine.hpp:171): a's elements rounded to out's width."""
        if a.complex != out.complex or a.count != out.count or not a.bits or not out.bits:
            raise InvalidArgument("cast buffers must have the same count and format")
        check(lib.lf_batch_cast(self.handle, a.bits, out.bits, int(a.complex), a.handle, out.handle, a.count))

    def tree_sum(self, a: Buffer, out: Buffer) -> None:
        """CommandBatch::tree_sum (engine.hpp:150): the adjacent-pair tree sum of a into out[0]."""
        if out.count != 1:
            raise InvalidArgument("tree_sum output must contain one element")
        if a.bits != out.bits or a.complex != out.complex:
            raise InvalidArgument("tree_sum buffers must have the same format")
        check(lib.lf_batch_tree_sum(self.handle, a.bits, int(a.complex), a.handle, out.handle, a.count))

    def submit(self) -> Submission:
        h = C.c_void_p()
        check(lib.lf_batch_submit(self.handle, C.byref(h)))
        done, self._completions = self._completions, []
        return Submission(h, done)


class Engine:
    """One CUDA device (engine.hpp:184-227).  One Engine per host thread."""

    def __init__(self, device: int = 0):
        opts = _EngineOptions(0, 1, 1, device)
        h = C.c_void_p()
        check(lib.lf_engine_create(C.byref(opts), C.byref(h)))
        self.handle = h

    def __del__(self):
        if getattr(self, "handle", None) and lib is not None:
            lib.lf_engine_destroy(self.handle)
            self.handle = None

    def device_name(self) -> str:
        buf = C.create_string_buffer(256)
        check(lib.lf_engine_device_name(self.handle, buf, 256))
        return buf.value.decode()

    def make_buffer(self, count: int, bits: int = 0, complex_: bool = False) -> Buffer:
        if bits:
            check_bits(bits)
        return Buffer(self, count, bits, complex_)

    def batch(self) -> CommandBatch:
        return CommandBatch(self)

    def run(self, bits, op, a, b, count=None, b_index: Broadcast | None = None, out=None):
        n = _elements(a) if count is None else count
        out = np.empty_like(a[:n]) if out is None else out
        t = _Timing()
        check(lib.lf_engine_run(self.handle, bits, int(op), _ptr(a), _ptr(b), _ptr(out), n, _bc(b_index), C.byref(t)))
        return out, _timing(t)

    def run_unary(self, bits, op, a, count=None, out=None):
        n = _elements(a) if count is None else count
        out = np.empty_like(a[:n]) if out is None else out
        t = _Timing()
        check(lib.lf_engine_run_unary(self.handle, bits, int(op), _ptr(a), _ptr(out), n, C.byref(t)))
        return out, _timing(t)

    def run_ternary(self, bits, op, a, b, c, count=None, b_index=None, c_index=None, out=None):
        n = _elements(a) if count is None else count
        out = np.empty_like(a[:n]) if out is None else out
        t = _Timing()
        check(lib.lf_engine_run_ternary(self.handle, bits, int(op), _ptr(a), _ptr(b), _ptr(c), _ptr(out), n,
                                        _bc(b_index), _bc(c_index), C.byref(t)))
        return out, _timing(t)

    def cast(self, from_bits, to_bits, complex_, x):
        """Engine::cast (engine.hpp:205), host arrays; returns (out, Timing)."""
        count = _elements(x)
        n = to_bits // 32
        out = np.zeros((count, 2, n + 3) if complex_ else (count, n + 3), dtype=np.uint32)
        t = _Timing()
        check(lib.lf_engine_cast(self.handle, from_bits, to_bits, int(complex_), _ptr(np.ascontiguousarray(x)), _ptr(out), count,
                                 C.byref(t)))
        return out, _timing(t)

    def segmented_dot(self, bits, complex_, shape: SegmentedDot, a, b):
        """Engine::segmented_dot (engine.hpp:205): returns (out [segments], Timing)."""
        n = check_bits(bits)
        out = np.zeros((shape.segments, 2, n + 3) if complex_ else (shape.segments, n + 3), dtype=np.uint32)
        sh = _SegmentedDot(shape.segments, shape.length, int(shape.shared_right))
        t = _Timing()
        check(lib.lf_engine_segmented_dot(self.handle, bits, int(complex_), C.byref(sh), _ptr(a), _ptr(b), _ptr(out), C.byref(t)))
        return out, _timing(t)

    def recurrence(self, bits, seeds, weights, count, steps, states_per_weight=1):
        """Engine::recurrence (engine.hpp:218-223): returns (out [count] complex, Timing)."""
        n = check_bits(bits)
        out = np.zeros((count, 2, n + 3), dtype=np.uint32)
        t = _Timing()
        check(lib.lf_engine_recurrence(self.handle, bits, _ptr(seeds), _ptr(weights), _ptr(out), count, steps, states_per_weight,
                                       C.byref(t)))
        return out, _timing(t)

    def lu4(self, bits, shape: Batched4, A, B=None):
        n = check_bits(bits)
        R = 4 if shape.inverse else shape.rhs
        X = np.zeros((shape.count * 4 * R, 2, n + 3), dtype=np.uint32)
        det = np.zeros((shape.count, 2, n + 3), dtype=np.uint32)
        st = np.zeros(shape.count, dtype=np.uint32)
        s = _Batched4(shape.count, shape.rhs, int(shape.inverse), int(shape.determinant), int(shape.fused))
        t = _Timing()
        check(lib.lf_engine_lu4(self.handle, bits, C.byref(s), _ptr(A), _ptr(B), _ptr(X), _ptr(det), _ptr(st), C.byref(t)))
        return X, det, st, _timing(t)


class ExactGemm4Ticket:
    """experimental::ExactGemm4Ticket (prototype.hpp:9-16): resolved once the batch's submission has been waited for."""

    def __init__(self, report: ExactGemm4Report):
        self._report = report
        self._done = False

    def resolved(self) -> bool:
        return self._done

    def report(self) -> ExactGemm4Report:
        if not self._done:
            raise LogicError("exact GEMM4: wait for submission before reading report")
        return self._report


class ExactGemm4:
    """experimental::ExactGemm4 (prototype.hpp:21-33): batches of row-major 4 x 4 products, each real component
    RN(C_old + sum of exact signed products), then optionally negated; complex components sum eight real products with
    one rounding.  Every component is summed exactly on the GPU, so no host repair is ever pending and outputs read later
    in the same batch are final."""

    def __init__(self, engine: "Engine"):
        self.engine = engine

    @staticmethod
    def _shape(s: ExactGemm4Shape) -> _ExactGemm4Shape:
        return _ExactGemm4Shape(s.count, s.stride_a, s.stride_b, s.stride_c, int(s.accumulate), int(s.negative))

    def gemm(self, bits, complex_, shape: ExactGemm4Shape, a, b, c):
        """Host arrays (prototype.hpp:32): c is updated in place; returns (Timing, ExactGemm4Report)."""
        if not (isinstance(c, np.ndarray) and c.flags.c_contiguous and c.dtype == np.uint32):
            raise InvalidArgument("exact_gemm4 output must be a C-contiguous uint32 array")
        r, t = _ExactGemm4Report(), _Timing()
        check(lib.lf_engine_exact_gemm4(self.engine.handle, bits, int(complex_), C.byref(self._shape(shape)),
                                        _ptr(np.ascontiguousarray(a)), _ptr(np.ascontiguousarray(b)), _ptr(c), C.byref(r), C.byref(t)))
        return _timing(t), ExactGemm4Report(r.gpu_components, r.host_components, bool(r.provisional_reads))

    def encode(self, batch: CommandBatch, shape: ExactGemm4Shape, a: Buffer, b: Buffer, c: Buffer) -> ExactGemm4Ticket:
        """Resident buffers recorded into batch (prototype.hpp:28-30)."""
        if not a.bits or a.bits != b.bits or a.bits != c.bits or a.complex != b.complex or a.complex != c.complex:
            raise InvalidArgument("exact_gemm4 buffers must share one arithmetic format")
        check(lib.lf_batch_exact_gemm4(batch.handle, a.bits, int(a.complex), C.byref(self._shape(shape)), a.handle, b.handle,
                                       c.handle))
        ticket = ExactGemm4Ticket(ExactGemm4Report(shape.count * 16 * (2 if a.complex else 1), 0, False))
        batch._completions.append(lambda: setattr(ticket, "_done", True))
        return ticket


class BatchedLinalg:
    """Sequential batched products (batched_linalg.hpp:63-118)."""

    def __init__(self, engine: Engine):
        self.engine = engine
        self._spaces: list = []

    @staticmethod
    def _shape(s: StridedGemm) -> _StridedGemm:
        return _StridedGemm(s.count, s.m, s.n, s.k, s.stride_a, s.stride_b, s.stride_c, int(s.accumulate), int(s.fused),
                            int(s.negative))

    def gemm(self, bits, complex_, s: StridedGemm, A, B, C_):
        """Host form: C_ is read and overwritten in place; returns Timing."""
        t = _Timing()
        sh = self._shape(s)
        check(lib.lf_batched_gemm(self.engine.handle, bits, int(complex_), C.byref(sh), _ptr(A), _ptr(B), _ptr(C_), C.byref(t)))
        return _timing(t)

    def gemm_resident(self, batch: CommandBatch, s: StridedGemm, A: Buffer, B: Buffer, C_: Buffer) -> None:
        sh = self._shape(s)
        check(lib.lf_batch_strided_gemm(batch.handle, A.bits, int(A.complex), C.byref(sh), A.handle, B.handle, C_.handle))

    def import_inline_complex(self, batch: CommandBatch, allocation: np.ndarray, records: np.ndarray, out: Buffer) -> None:
        """BatchedLinalg::import_inline_complex (batched_linalg.hpp:146-148): out[i] gathered on the GPU from the MPFR
        significands inside `allocation` (whole aligned pages, see page_aligned) that records[i] (INLINE_RECORD_DTYPE)
        describes.  The allocation must stay unchanged until the batch has been submitted."""
        if not out.complex or not out.bits:
            raise InvalidArgument("inline complex staging needs complex output")
        if records.dtype != INLINE_RECORD_DTYPE or not records.flags.c_contiguous:
            raise InvalidArgument("records must be a contiguous INLINE_RECORD_DTYPE array")
        if out.count < len(records):
            raise InvalidArgument("inline staging: undersized buffer")
        check(lib.lf_batch_import_inline_complex(batch.handle, out.bits, allocation.ctypes.data, allocation.nbytes,
                                                 records.ctypes.data if len(records) else None, len(records), out.handle))
        batch._completions.append(lambda keep=(allocation, records): None)   # both stay referenced until the wait

    def product3(self, batch: CommandBatch, first: StridedGemm, second: StridedGemm, A: Buffer, B: Buffer, D: Buffer, C_: Buffer,
                 negative=False) -> None:
        """C_b = (A_b B_b) D_b (batched_linalg.hpp:99-110) through an intermediate kept by this BatchedLinalg."""
        import dataclasses
        if first.count != second.count or first.m != second.m or first.n != second.k or first.accumulate or second.accumulate:
            raise InvalidArgument("product3: incompatible shapes or accumulation")
        first = dataclasses.replace(first, stride_c=first.m * first.n)
        second = dataclasses.replace(second, stride_a=first.m * first.n, negative=bool(negative))
        count = max(first.count * first.stride_c, 1)
        tmp = next((b for b in self._spaces if b.bits == A.bits and b.complex == A.complex and b.count >= count
                    and lib.lf_buffer_holders(b.handle) == 0), None)
        if tmp is None:
            tmp = self.engine.make_buffer(count, A.bits, A.complex)
            self._spaces.append(tmp)
        self.gemm_resident(batch, first, A, B, tmp)
        self.gemm_resident(batch, second, tmp, D, C_)

    def workspaces(self) -> dict:
        """product3 intermediates: idle (held by no batch or unwaited submission) and busy bytes."""
        w = {"idle_bytes": 0, "busy_bytes": 0, "busy_workspaces": 0}
        for b in self._spaces:
            size = 4 * b.words * b.count
            if lib.lf_buffer_holders(b.handle) == 0:
                w["idle_bytes"] += size
            else:
                w["busy_bytes"] += size
                w["busy_workspaces"] += 1
        return w

    def release_workspaces(self) -> dict:
        w = self.workspaces()
        self._spaces = []
        return w


@dataclass
class RaggedLu4:
    """The batched 4x4 LU job of a ragged plan: Engine::lu4 semantics (engine.hpp:164) on arena data."""
    bits: int
    shape: Batched4
    A: int = 0
    B: int = 0
    X: int = 0
    det: int = 0
    status: int = 0

    def _c(self) -> _RaggedLu4:
        s = self.shape
        return _RaggedLu4(self.bits, _Batched4(s.count, s.rhs, int(s.inverse), int(s.determinant), int(s.fused)),
                          self.A, self.B, self.X, self.det, self.status)


def ragged_items(bits, m, n, k, accumulate=0, negative=0) -> np.ndarray:
    """Instance table (RAGGED_DTYPE) from per-instance arrays; offsets are filled by ragged_pack."""
    bits = np.asarray(bits)
    t = np.zeros(bits.shape[0], RAGGED_DTYPE)
    t["bits"], t["m"], t["n"], t["k"] = bits, m, n, k
    t["accumulate"], t["negative"] = accumulate, negative
    return t


def ragged_pack(complex_: bool, items: np.ndarray, lu4: "RaggedLu4 | None" = None) -> int:
    """Assigns packed byte offsets in place (and the LU job's); returns the arena size in bytes."""
    if items.dtype != RAGGED_DTYPE or not items.flags["C_CONTIGUOUS"]:
        raise InvalidArgument("items must be a contiguous RAGGED_DTYPE array")
    total = C.c_uint64()
    cl = lu4._c() if lu4 is not None else None
    check(lib.lf_ragged_pack(int(complex_), _ptr(items), items.shape[0], C.byref(cl) if cl is not None else None,
                             C.byref(total)))
    if lu4 is not None:
        lu4.A, lu4.B, lu4.X, lu4.det, lu4.status = cl.A, cl.B, cl.X, cl.det, cl.status
    return int(total.value)


class RaggedPlan:
    """A ragged mixed-precision batch over one device arena, run as one CUDA graph launch
    (lf_ragged_plan_*; no reference counterpart)."""

    def __init__(self, engine: Engine, complex_: bool, fused: bool, items: np.ndarray, arena_bytes: int,
                 lu4: "RaggedLu4 | None" = None):
        if items.dtype != RAGGED_DTYPE or not items.flags["C_CONTIGUOUS"]:
            raise InvalidArgument("items must be a contiguous RAGGED_DTYPE array")
        self.engine = engine
        h = C.c_void_p()
        cl = lu4._c() if lu4 is not None else None
        check(lib.lf_ragged_plan_create(engine.handle, int(complex_), int(fused), _ptr(items), items.shape[0],
                                        C.byref(cl) if cl is not None else None, int(arena_bytes), C.byref(h)))
        self.handle = h

    def tune(self, arena_ptr: int) -> None:
        check(lib.lf_ragged_plan_tune(self.handle, C.c_void_p(arena_ptr)))

    def run(self, arena_ptr: int, stream: int = 0) -> None:
        check(lib.lf_ragged_plan_run(self.handle, C.c_void_p(arena_ptr), C.c_void_p(stream)))

    def info(self) -> dict:
        i = _RaggedInfo()
        check(lib.lf_ragged_plan_get_info(self.handle, C.byref(i)))
        return {"tuned": bool(i.tuned), "lu4_block": i.lu4_block, "lu4_grid": i.lu4_grid, "lu4_trial_ms": i.lu4_trial_ms,
                "classes": [{"bits": c.bits, "items": c.items, "cells": c.cells, "block": c.block, "grid": c.grid,
                             "trial_ms": c.trial_ms} for c in i.cls[:i.classes]]}

    def __del__(self):
        if getattr(self, "handle", None) and lib is not None:
            lib.lf_ragged_plan_destroy(self.handle)
            self.handle = None


class PinnedArray:
    """numpy array over page-locked host memory (lf_host_alloc); freed with the object."""

    def __init__(self, shape, dtype=np.uint32):
        self.nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
        p = C.c_void_p()
        check(lib.lf_host_alloc(self.nbytes, C.byref(p)))
        self._p = p
        buf = (C.c_char * max(self.nbytes, 1)).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)

    def __del__(self):
        if getattr(self, "_p", None) and lib is not None:
            self.array = None
            lib.lf_host_free(self._p)
            self._p = None


class LinalgTicket:
    """Handle of a resident product (linalg.hpp:60-66)."""

    def __init__(self, handle):
        self.handle = handle

    def resolved(self) -> bool:
        r = C.c_int()
        check(lib.lf_linalg_ticket_resolved(self.handle, C.byref(r)))
        return bool(r.value)

    def report(self) -> dict:
        r = _LinalgReport()
        check(lib.lf_linalg_ticket_report(self.handle, C.byref(r)))
        return {f: getattr(r, f) for f, _ in _LinalgReport._fields_}

    def __del__(self):
        if getattr(self, "handle", None) and lib is not None:
            lib.lf_linalg_ticket_destroy(self.handle)
            self.handle = None


class Linalg:
    """Exact dense products and factorizations (linalg.hpp:141-218).  One Linalg per host thread."""

    def __init__(self, engine: "Engine | None" = None, options: LinalgOptions | None = None):
        o = options or LinalgOptions()
        self.options = o
        self.engine = engine
        co = _LinalgOptions(o.band_bits, o.max_bands, o.max_spread, o.host_threads, int(o.force_fallback),
                            o.resident_bands, o.method)
        h = C.c_void_p()
        check(lib.lf_linalg_create(engine.handle if engine else None, C.byref(co), C.byref(h)))
        self.handle = h

    def __del__(self):
        if getattr(self, "handle", None) and lib is not None:
            lib.lf_linalg_destroy(self.handle)
            self.handle = None

    def report(self) -> dict:
        r = _LinalgReport()
        check(lib.lf_linalg_get_report(self.handle, C.byref(r)))
        return {f: getattr(r, f) for f, _ in r._fields_}

    def workspaces(self) -> dict:
        """Device memory retained between calls (linalg.hpp:46-52, 179): scratch, idle and busy resident workspaces."""
        w = _LinalgWorkspaces()
        check(lib.lf_linalg_get_workspaces(self.handle, C.byref(w)))
        return {f: getattr(w, f) for f, _ in w._fields_}

    def release_workspaces(self) -> dict:
        """Frees the scratch and idle resident workspaces (linalg.hpp:173-180); returns what was retained before."""
        w = _LinalgWorkspaces()
        check(lib.lf_linalg_release_workspaces(self.handle, C.byref(w)))
        return {f: getattr(w, f) for f, _ in w._fields_}

    def gemm(self, bits, transpose_a, A, B, m, n, k, C_, subtract=False) -> Timing:
        t = _Timing()
        check(lib.lf_linalg_gemm(self.handle, bits, int(transpose_a), _ptr(A), _ptr(B), m, n, k, _ptr(C_), int(subtract),
                                 C.byref(t)))
        return _timing(t)

    def syrk(self, bits, A, rows, cols, C_, lower_only=True, subtract=False) -> Timing:
        t = _Timing()
        check(lib.lf_linalg_syrk(self.handle, bits, _ptr(A), rows, cols, _ptr(C_), int(lower_only), int(subtract), C.byref(t)))
        return _timing(t)

    @staticmethod
    def _fo(o: FactorOptions | None):
        o = o or FactorOptions()
        return _FactorOptions(o.block, o.host_macs, o.solve_host_macs, int(o.gpu))

    def cholesky(self, bits, A, n, L, options: FactorOptions | None = None) -> CholeskyInfo:
        i = _CholeskyInfo()
        fo = self._fo(options)
        check(lib.lf_linalg_cholesky(self.handle, bits, _ptr(A), n, _ptr(L), C.byref(fo), C.byref(i)))
        return CholeskyInfo(i.pivot, i.pivot_sign, i.pivot_status, _timing(i.timing), i.blocks, i.gpu_updates,
                            i.host_updates, i.panel_seconds, i.update_seconds)

    def trsm(self, bits, transpose, L, n, B, nrhs, X, options: FactorOptions | None = None) -> Timing:
        t = _Timing()
        fo = self._fo(options)
        check(lib.lf_linalg_trsm(self.handle, bits, int(transpose), _ptr(L), n, _ptr(B), nrhs, _ptr(X), C.byref(fo), C.byref(t)))
        return _timing(t)

    def cholesky_solve(self, bits, L, n, B, nrhs, X, options: FactorOptions | None = None) -> Timing:
        t = _Timing()
        fo = self._fo(options)
        check(lib.lf_linalg_cholesky_solve(self.handle, bits, _ptr(L), n, _ptr(B), nrhs, _ptr(X), C.byref(fo), C.byref(t)))
        return _timing(t)

    @staticmethod
    def _qo(o: "QROptions | None"):
        o = o or QROptions()
        return _QROptions(o.block, o.host_macs, o.solve_host_macs, int(o.gpu), o.rank_bits, int(o.pivot))

    def factor_qr(self, bits, A, m, n, options: "QROptions | None" = None) -> "QRFactor":
        """Householder QR of A (m x n, m >= n, row-major) (linalg.hpp:164); A is only read."""
        h = C.c_void_p()
        qo = self._qo(options)
        check(lib.lf_linalg_factor_qr(self.handle, bits, _ptr(A), m, n, C.byref(qo), C.byref(h)))
        return QRFactor(h, self)

    def factor_qr_augmented(self, bits, J, m, n, d, options: "QROptions | None" = None) -> "QRFactor":
        """The factor of [J; diag(d)] ((m + n) x n) (linalg.hpp:168)."""
        h = C.c_void_p()
        qo = self._qo(options)
        check(lib.lf_linalg_factor_qr_augmented(self.handle, bits, _ptr(J), m, n, _ptr(d), C.byref(qo), C.byref(h)))
        return QRFactor(h, self)

    def factor_qr_complex(self, bits, A, m, n, options: "QROptions | None" = None) -> "QRFactor":
        """Complex Householder QR of A (m x n complex, shape [m * n, 2, N + 3]) (linalg.hpp:170): H = I - tau v v^H with
        complex tau, R upper with a real diagonal.  Column pivoting of complex factors is not built."""
        h = C.c_void_p()
        qo = self._qo(options)
        check(lib.lf_linalg_factor_qr_complex(self.handle, bits, _ptr(A), m, n, C.byref(qo), C.byref(h)))
        return QRFactor(h, self)

    def factor_qr_buffer(self, A: "Buffer", m, n, options: "QROptions | None" = None) -> "QRFactor":
        """factor_qr on an idle Buffer of this Linalg's engine (linalg.hpp:200)."""
        h = C.c_void_p()
        qo = self._qo(options)
        check(lib.lf_linalg_factor_qr_buffer(self.handle, A.bits, A.handle, m, n, C.byref(qo), C.byref(h)))
        return QRFactor(h, self)

    # explicit contract names (linalg.hpp:203-210)
    gemm_exact = gemm
    syrk_exact = syrk
    cholesky_blocked = cholesky
    cholesky_solve_blocked = cholesky_solve

    # resident products (linalg.hpp:190-195): recorded into a batch, planned and run on the GPU at submit
    def gemm_resident(self, batch: "CommandBatch", transpose_a, A: "Buffer", B: "Buffer", m, n, k, C_: "Buffer",
                      subtract=False) -> "LinalgTicket":
        h = C.c_void_p()
        check(lib.lf_linalg_batch_gemm(self.handle, batch.handle, A.bits, int(transpose_a), A.handle, B.handle, m, n, k, C_.handle,
                                       int(subtract), C.byref(h)))
        return LinalgTicket(h)

    def syrk_resident(self, batch: "CommandBatch", A: "Buffer", rows, cols, C_: "Buffer", lower_only=True,
                      subtract=False) -> "LinalgTicket":
        h = C.c_void_p()
        check(lib.lf_linalg_batch_syrk(self.handle, batch.handle, A.bits, A.handle, rows, cols, C_.handle, int(lower_only),
                                       int(subtract), C.byref(h)))
        return LinalgTicket(h)

    def dev_exact_product(self, bits, left, left_ls, left_ks, right, right_ls, right_ks, M, N, K, C_, ldc,
                          subtract=False, lower=False, stream=0) -> None:
        check(lib.lf_dev_exact_product(self.handle, bits, _ptr(left), left_ls, left_ks, _ptr(right), right_ls, right_ks,
                                       M, N, K, _ptr(C_), ldc, int(subtract), int(lower), C.c_void_p(stream)))


class QRFactor:
    """Owning Householder QR factor (linalg.hpp:109-138): Q = H_0 ... H_{n-1}, H_j = I - tau_j v_j v_j^T, and R.  Uses
    the Linalg that made it (kept alive here)."""

    def __init__(self, handle, linalg: Linalg):
        self.handle = handle
        self.linalg = linalg
        bits, rows, cols, block, piv = C.c_int(), C.c_size_t(), C.c_size_t(), C.c_size_t(), C.c_int()
        i = _QRInfo()
        check(lib.lf_qr_describe(handle, C.byref(bits), C.byref(rows), C.byref(cols), C.byref(block), C.byref(piv), C.byref(i)))
        self.bits, self.rows, self.cols, self.block, self.pivoted = bits.value, rows.value, cols.value, block.value, bool(piv.value)
        self.complex = bool(lib.lf_qr_is_complex(handle))
        self.info = QRInfo(i.rank, i.reason, i.status, _timing(i.timing), i.blocks, i.gpu_updates, i.host_updates,
                           i.panel_seconds, i.update_seconds, i.norm_recomputations)

    def __del__(self):
        if getattr(self, "handle", None) and lib is not None:
            lib.lf_qr_destroy(self.handle)
            self.handle = None

    def full_rank(self) -> bool:
        return self.info.rank == self.cols

    def _array(self, fn, count) -> np.ndarray:
        w = self.bits // 32 + 3
        shape = (count, 2, w) if self.complex else (count, w)
        p = fn(self.handle)                      # R, V and T are copied from the device on the first call
        if not count:
            return np.zeros((0,) + shape[1:], dtype=np.uint32)
        if not p:
            raise RuntimeFailure("QR factor arrays: " + lib.lf_last_error().decode())
        total = count * w * (2 if self.complex else 1)
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint32)), shape=(total,)).reshape(shape).copy()

    def r(self) -> np.ndarray:
        return self._array(lib.lf_qr_r, self.cols * self.cols)

    def v(self) -> np.ndarray:
        return self._array(lib.lf_qr_v, self.rows * self.cols)

    def tau(self) -> np.ndarray:
        return self._array(lib.lf_qr_tau, self.cols)

    def t(self) -> np.ndarray:
        nb = self.block
        blocks = (self.cols + nb - 1) // nb if nb else 0
        return self._array(lib.lf_qr_t, blocks * nb * nb)

    def permutation(self) -> list:
        p = lib.lf_qr_permutation(self.handle)
        return [int(p[i]) for i in range(self.cols)] if self.cols else []

    def solve(self, B, nrhs, X=None) -> np.ndarray:
        """Least-squares X (n x nrhs) for B (m x nrhs) (linalg.hpp:127)."""
        if X is None:
            w = self.bits // 32 + 3
            X = np.zeros((self.cols * nrhs, 2, w) if self.complex else (self.cols * nrhs, w), dtype=np.uint32)
        t = _Timing()
        check(lib.lf_qr_solve(self.handle, _ptr(B), nrhs, _ptr(X), C.byref(t)))
        self.last_timing = _timing(t)
        return X

    def apply_q(self, B, nrhs, transpose) -> Timing:
        """B (m x nrhs) <- Q^T B (transpose) or Q B, in place (linalg.hpp:129)."""
        t = _Timing()
        check(lib.lf_qr_apply_q(self.handle, _ptr(B), nrhs, int(bool(transpose)), C.byref(t)))
        return _timing(t)

    def solve_buffers(self, B: "Buffer", nrhs, X: "Buffer") -> Timing:
        t = _Timing()
        check(lib.lf_qr_solve_buffers(self.handle, B.handle, nrhs, X.handle, C.byref(t)))
        return _timing(t)

    def apply_q_buffer(self, B: "Buffer", nrhs, transpose) -> Timing:
        t = _Timing()
        check(lib.lf_qr_apply_q_buffer(self.handle, B.handle, nrhs, int(bool(transpose)), C.byref(t)))
        return _timing(t)


def dev_elementwise(bits, op, a_ptr, b_ptr, c_ptr, out_ptr, count, b_index=None, c_index=None, stream=0) -> None:
    check(lib.lf_dev_elementwise(bits, int(op), _ptr(a_ptr), _ptr(b_ptr), _ptr(c_ptr), _ptr(out_ptr), count,
                                 _bc(b_index), _bc(c_index), C.c_void_p(stream)))


def dev_mul_chain(bits, x_ptr, factors_ptr, factor_stride, steps, out_ptr, count, stream=0) -> None:
    check(lib.lf_dev_mul_chain(bits, _ptr(x_ptr), _ptr(factors_ptr), factor_stride, steps, _ptr(out_ptr), count,
                               C.c_void_p(stream)))


def dev_mul_chain_lanes(bits, lanes, x_ptr, factors_ptr, factor_stride, steps, out_ptr, count, stream=0) -> None:
    check(lib.lf_dev_mul_chain_lanes(bits, lanes, _ptr(x_ptr), _ptr(factors_ptr), factor_stride, steps, _ptr(out_ptr), count,
                                     C.c_void_p(stream)))


def dev_cast(from_bits, to_bits, complex_, in_ptr, out_ptr, count, stream=0) -> None:
    check(lib.lf_dev_cast(from_bits, to_bits, int(complex_), C.c_void_p(in_ptr), C.c_void_p(out_ptr), count, C.c_void_p(stream)))


def dev_tree_sum(bits, complex_, in_ptr, count, out_ptr, scratch_ptr, stream=0) -> None:
    """scratch: 2 * ceil(count / 2) elements (unused for count <= 2)."""
    check(lib.lf_dev_tree_sum(bits, int(complex_), C.c_void_p(in_ptr), count, C.c_void_p(out_ptr),
                              C.c_void_p(scratch_ptr), C.c_void_p(stream)))


def word_mac_rate(device: int = 0) -> float:
    """Measured rate of 32 x 32 -> 64-bit integer multiply-adds on `device` (lf_probe_word_mac_rate)."""
    r = C.c_double()
    check(lib.lf_probe_word_mac_rate(device, C.byref(r)))
    return r.value


def residue_wait_limit_test(polls: int) -> int:
    """Failure-detection hook: a residue-product tile whose first barrier wait runs out after `polls` polls;
    returns the kernel's error word (2 when the bounded wait gave up)."""
    e = C.c_uint32()
    check(lib.lf_test_residue_wait_limit(polls, C.byref(e)))
    return e.value
