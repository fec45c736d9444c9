"""Benchmark of the headline workload: bit-exact 1024-bit (32-limb) 16-step multiplication
chains over 65,536 values, every step rounded to nearest-even (the resident chain of the
reference's CommandBatch::run(mul, x, f_s, x) x16, engine.mm:332-346).

One step = one pass of the chain over the whole batch = 1,048,576 rounded 1024-bit products.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

``value``   device throughput: inputs resident in HBM, CUDA events on the launching stream.
``e2e``     the same through the public API (Engine / Buffer / CommandBatch): pinned host arrays
            uploaded, 16 resident muls submitted and waited, the result downloaded, per step.
``--impl reference`` times the reference's own CPU implementation (its core.hpp compiled from
the reference sources into oracle/_ref, or the C oracle where that build is absent) on all
host cores over a bounded sample of the same workload.
Under torchrun (N > 1) every rank runs its own 65,536-value chain (weak scaling; the path has
no exchange step), times it on its device and rank 0 reports the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BITS, COUNT, CHAIN = 1024, 65536, 16
METRIC = "1024-bit ops/s; exact GEMM MAC/s int8-CRT vs limb kernel, 1 B200, bit-exact"
UNIT = "1024-bit ops/s"
WORKLOAD = "1024-bit (32-limb) 16-step RNE multiplication chains over 65,536 values"
ELEMENT_BYTES = BITS // 8 + 12
# ncu: dram__bytes_read.sum + dram__bytes_write.sum of one launch of the 1024-bit chain kernel on this
# workload, from one capture (156,188,928 + 4,269,568 bytes).
TRAFFIC_BYTES = 160458496


# word products of the upper-half 1024-bit product (every a_i b_j with i + j >= N - 2 at N = 32 limbs)
UPPER_PRODUCTS = sum(1 for i in range(32) for j in range(32) if i + j >= 30)


def make_inputs(seed: int = 20261203):
    """Seeded synthetic data of the chain workload: significands uniform with the
    top bit set, exponents uniform in [-8, 8], 1% exact zeros, 2% sparse significands."""
    from limbforge_b200 import numbers as nb
    rng = np.random.default_rng(seed)
    x = nb.random_numbers(rng, COUNT, BITS, 8, zero_frac=0.01, sparse_frac=0.02)
    f = np.stack([nb.random_numbers(rng, COUNT, BITS, 8, zero_frac=0.01, sparse_frac=0.02) for _ in range(CHAIN)])
    return x, f


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML every 5 ms while running."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, device: int):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                break
            time.sleep(0.005)

    def __enter__(self):
        if self.nv:
            self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self.nv:
            self._t.join()

    def summary(self):
        return {"sm_mhz": float(np.median(self.samples)) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_reference_rate(x, f, sample: int, threads: int | None = None):
    """The reference's CPU chain (its core.hpp mul, or the C oracle where the reference build
    is absent) over `sample` values on all host cores; returns (ops/s, kind, cores)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle.oracle import Oracle, Reference
    threads = threads or os.cpu_count() or 1
    xs = np.ascontiguousarray(x[:sample])
    fs = np.ascontiguousarray(f[:, :sample])
    if Reference.available():
        ref, kind = Reference(), "reference"

        def work(lo, hi):
            v = np.ascontiguousarray(xs[lo:hi])
            for s in range(CHAIN):
                v = ref.elementwise(BITS, 2, v, np.ascontiguousarray(fs[s, lo:hi]))
            return v
        chunks = np.linspace(0, sample, threads + 1).astype(int)
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(lambda i: work(chunks[i], chunks[i + 1]), range(threads)))
        dt = time.perf_counter() - t0
    else:
        orc, kind = Oracle(), "port"
        t0 = time.perf_counter()
        orc.mul_chain(BITS, xs, fs)
        dt = time.perf_counter() - t0
    return sample * CHAIN / dt, kind, threads


def mpfr_chain_rates(x, f, gpu_result=None):
    """The MPFR baseline the reference's benchmarks use (benchmarks/benchmark.cpp:3-94): the whole workload
    (every value, 16 steps, mpfr_mul at 1024 bits RNDN over preallocated mpfr_t), serial and on one worker per
    host core, 2 warm-up and 9 timed passes each, alternating; median pass rates, and whether the MPFR values
    equal the GPU's bit for bit."""
    try:
        from oracle.oracle import Mpfr
        threads = os.cpu_count() or 1
        times, out = Mpfr().chain_baseline(BITS, x, np.ascontiguousarray(f), [1, threads])
    except Exception as e:                                   # reported, never hidden
        return {"error": f"{type(e).__name__}: {e}"}
    ops = x.shape[0] * f.shape[0]
    r = {"serial_ops_per_s": ops / times[1], "all_core_ops_per_s": ops / times[threads], "cores": threads,
         "unit": UNIT, "sample": f"all {x.shape[0]} values x {f.shape[0]} steps, median of 9 passes"}
    if gpu_result is not None:
        r["bit_exact_vs_gpu"] = bool((out == gpu_result).all())
    return r


def word_mac_peak(api, device):
    try:
        return api.word_mac_rate(device)
    except Exception:
        return None


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path on the host cores, rank 0 only."""
    if rank != 0:
        return
    x, f = make_inputs()
    sample = int(os.environ.get("LF_CPU_SAMPLE", "8192"))
    rates = []
    for i in range(args.warmup + args.steps):
        r, kind, cores = cpu_reference_rate(x, f, sample)
        if i >= args.warmup:
            rates.append(r)
    value = float(np.median(rates))
    mpfr = mpfr_chain_rates(x, f)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": COUNT * CHAIN / value * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 limbs (1024-bit RNE)", "data": "synthetic",
        "config": {"workload": WORKLOAD, "count": COUNT, "steps_per_chain": CHAIN, "bits": BITS},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{sample} of {COUNT} values x {CHAIN} steps per step, extrapolated"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "mpfr": mpfr,
    }), flush=True)


# ---------------------------------------------------------------- secondary workloads
# Secondary measurements printed inside the same JSON line under "workloads" (1 GPU only): each one
# is timed on device-resident data and checked against the oracle on a sample.

def _log(msg):
    print(f"[bench] {msg}", file=sys.stderr, flush=True)


def _event_ms(torch, stream, fn, reps):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _threads_rate(fn, total, threads):
    """Runs fn(lo, hi) over [0, total) split across host threads; returns seconds."""
    from concurrent.futures import ThreadPoolExecutor
    cuts = np.linspace(0, total, threads + 1).astype(int)
    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(lambda i: fn(cuts[i], cuts[i + 1]), range(threads)))
    return time.perf_counter() - t0


def elementwise_256(torch, api, hbm_peak):
    """256-bit RNE mul, div and fma on 65,536 elements (exponents U[-256,256], 1% zeros, 2% sparse)."""
    from limbforge_b200 import numbers as nb
    from oracle.oracle import Oracle, Reference
    bits, cnt = 256, 65536
    rng = np.random.default_rng(100)
    a, b, c = (nb.random_numbers(rng, cnt, bits, 256, zero_frac=0.01, sparse_frac=0.02) for _ in range(3))
    da, db, dc = (torch.from_numpy(x.view(np.int32)).cuda() for x in (a, b, c))
    do = torch.empty_like(da)
    st = torch.cuda.Stream()
    orc = Oracle()
    ref = Reference() if Reference.available() else None
    threads = os.cpu_count() or 1
    out = {}
    for op, name, nin in ((2, "mul", 2), (3, "div", 2), (9, "fma", 3)):
        def go():
            api.dev_elementwise(bits, op, da.data_ptr(), db.data_ptr(), dc.data_ptr() if nin == 3 else None, do.data_ptr(), cnt,
                                stream=st.cuda_stream)
        for _ in range(5):
            go()
        ms = _event_ms(torch, st, go, 200)
        got = do.cpu().numpy().view(np.uint32)
        want = orc.elementwise(bits, op, a, b, c if nin == 3 else None)
        moved = cnt * nb.element_bytes(bits) * (nin + 1)
        cpu = None
        if ref is not None:
            dt = _threads_rate(lambda lo, hi: ref.elementwise(bits, op, np.ascontiguousarray(a[lo:hi]), np.ascontiguousarray(b[lo:hi]),
                                                              np.ascontiguousarray(c[lo:hi]) if nin == 3 else None), cnt, threads)
            cpu = {"ops_per_s": cnt / dt, "cores": threads, "kind": "reference"}
        out[name] = {"us": ms * 1e3, "ops_per_s": cnt / (ms * 1e-3), "GB_per_s": moved / (ms * 1e-3) / 1e9,
                     "hbm_frac": moved / (ms * 1e-3) / 1e9 / hbm_peak, "bit_exact": bool((got == want).all()),
                     "cpu_reference": cpu}
    # the same mul at growing counts: per-launch overhead against HBM streaming
    sweep = []
    for cnt2 in (1 << 16, 1 << 18, 1 << 20, 1 << 22):
        a2 = torch.randint(0, 2**31 - 1, (cnt2, bits // 32 + 3), dtype=torch.int32, device="cuda")
        a2[:, bits // 32 - 1] |= -2**31
        a2[:, bits // 32] = 0
        a2[:, bits // 32 + 1] = 1
        a2[:, bits // 32 + 2] = 0
        o2 = torch.empty_like(a2)

        def go2():
            api.dev_elementwise(bits, 2, a2.data_ptr(), a2.data_ptr(), None, o2.data_ptr(), cnt2, stream=st.cuda_stream)
        for _ in range(3):
            go2()
        ms2 = _event_ms(torch, st, go2, 50)
        moved2 = cnt2 * nb.element_bytes(bits) * 3
        sweep.append({"count": cnt2, "us": ms2 * 1e3, "GB_per_s": moved2 / (ms2 * 1e-3) / 1e9,
                      "hbm_frac": moved2 / (ms2 * 1e-3) / 1e9 / hbm_peak})
        del a2, o2
    out["mul_count_sweep"] = sweep
    out["workload"] = "256-bit mul/div/fma, 65,536 elements per operand, device resident (launch-latency bound at this size)"
    return out


def cdiv_1024(torch, api):
    """1024-bit complex division on 65,536 pairs (components as the chain's values)."""
    from limbforge_b200 import numbers as nb
    from oracle.oracle import Oracle
    bits, cnt = 1024, 65536
    rng = np.random.default_rng(101)
    x = nb.random_complex(rng, cnt, bits, 8, zero_frac=0.01, sparse_frac=0.02)
    y = nb.random_complex(rng, cnt, bits, 8, zero_frac=0.01, sparse_frac=0.02)
    dx, dy = (torch.from_numpy(v.view(np.int32)).cuda() for v in (x, y))
    dz = torch.empty_like(dx)
    st = torch.cuda.Stream()

    def go():
        api.dev_elementwise(bits, 6, dx.data_ptr(), dy.data_ptr(), None, dz.data_ptr(), cnt, stream=st.cuda_stream)
    for _ in range(3):
        go()
    ms = _event_ms(torch, st, go, 20)
    got = dz.cpu().numpy().view(np.uint32)
    want = Oracle().elementwise(bits, 6, x, y)
    return {"workload": "1024-bit complex division, 65,536 pairs", "ms": ms, "pairs_per_s": cnt / (ms * 1e-3),
            "cdiv_full_match": bool((got == want).all()), "checked": cnt}


def exact_gemm_512(torch, api, scale=1.0):
    """512-bit C <- RN(C - A^T B), A, B 1024 x 1024 (exponents U[-40,40], 0.5% zeros), residue engine
    vs the plain limb kernel on the same device data; SYRK A^T A (lower).  `scale` shrinks n (profiling)."""
    from limbforge_b200 import numbers as nb
    from oracle.oracle import Oracle, Reference
    bits, n = 512, max(128, int(1024 * scale) // 128 * 128)
    rng = np.random.default_rng(102)
    A = nb.random_numbers(rng, n * n, bits, 40, zero_frac=0.005)
    B = nb.random_numbers(rng, n * n, bits, 40, zero_frac=0.005)
    C0 = nb.random_numbers(rng, n * n, bits, 40, zero_frac=0.005)
    dA, dB, dC0 = (torch.from_numpy(v.view(np.int32)).cuda() for v in (A, B, C0))
    eng = api.Engine()
    la = {m: api.Linalg(eng, api.LinalgOptions(method=m)) for m in (1, 2)}
    res, outs = {}, {}
    for m, name in ((2, "residue"), (1, "limb")):
        dC = dC0.clone()
        reps = 3 if m == 2 else 1
        times = []
        for r in range(reps + 1):
            dC.copy_(dC0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            la[m].dev_exact_product(bits, dA.data_ptr(), 1, n, dB.data_ptr(), 1, n, n, n, n, dC.data_ptr(), n, subtract=True)
            torch.cuda.synchronize()
            if r:
                times.append(time.perf_counter() - t0)
        t = float(np.median(times))
        outs[name] = dC
        res[name] = {"s": t, "mac_per_s": n ** 3 / t, "report": la[m].report()}
    res["identical_bits"] = bool(torch.equal(outs["residue"], outs["limb"]))
    res["speedup_residue_vs_limb"] = res["limb"]["s"] / res["residue"]["s"]
    rep = res["residue"]["report"]
    kp = (n + 127) // 128 * 128
    int8_macs = 4 * rep["moduli"] * kp * kp * kp
    res["residue"]["int8_tops_whole_call"] = 2 * int8_macs / res["residue"]["s"] / 1e12
    # oracle on one full output row
    got = outs["residue"].cpu().numpy().view(np.uint32)
    row = 517 % n
    want = Oracle().gemm(bits, True, A, B, n, n, n, C=C0, subtract=True, rows=(row, row + 1))
    res["oracle_row_match"] = bool((got[row * n:(row + 1) * n] == want[row * n:(row + 1) * n]).all())
    # SYRK A^T A lower, residue engine
    dS = torch.zeros_like(dC0)
    times = []
    for r in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        la[2].dev_exact_product(bits, dA.data_ptr(), 1, n, dA.data_ptr(), 1, n, n, n, n, dS.data_ptr(), n, lower=True)
        torch.cuda.synchronize()
        if r:
            times.append(time.perf_counter() - t0)
    ts = float(np.median(times))
    res["syrk_residue"] = {"s": ts, "mac_per_s": n * n * (n + 1) / 2 / ts}
    # the reference's exact_dot_add on all host cores over sampled outputs
    if Reference.available():
        ref = Reference()
        At = np.ascontiguousarray(A.reshape(n, n, -1).transpose(1, 0, 2))        # column i of A as a row
        Bt = np.ascontiguousarray(B.reshape(n, n, -1).transpose(1, 0, 2))
        sample = 256
        idx = rng.integers(0, n, size=(sample, 2))
        threads = os.cpu_count() or 1

        def work(lo, hi):
            for i, j in idx[lo:hi]:
                ref.exact_dot_add(bits, C0[i * n + j], True, At[i], 1, Bt[j], 1, n)
        dt = _threads_rate(work, sample, threads)
        res["cpu_reference"] = {"mac_per_s": sample * n / dt, "cores": threads, "kind": "reference",
                                "sample": f"{sample} outputs of {n * n}"}
    res["workload"] = "512-bit exact GEMM C <- RN(C - A^T B), 1024 x 1024 x 1024, device-pointer entry, synchronous call"
    return res


def cholesky_2048(torch, api):
    """256-bit SPD A = RN(G^T G) + n I (n = 2048, G uniform in [-1, 1]), blocked Cholesky (block 32),
    64 right-hand sides; scaled residual ||B - A X|| / (||A|| ||X||) from an exact residual product."""
    from limbforge_b200 import numbers as nb
    from oracle.oracle import Oracle
    bits, n, nrhs = 256, 2048, 64
    rng = np.random.default_rng(103)

    def uniform(count):
        x = nb.random_numbers(rng, count, bits, 0)
        x[:, bits // 32] = (-rng.geometric(0.5, size=count)).astype(np.int32).view(np.uint32)
        return x
    G = uniform(n * n)
    eng = api.Engine()
    la = api.Linalg(eng)
    A = np.zeros_like(G)
    t0 = time.perf_counter()
    la.syrk(bits, G, n, n, A, lower_only=False)
    t_syrk = time.perf_counter() - t0
    diag = np.ascontiguousarray(A[np.arange(n) * (n + 1)])
    nn = nb.random_numbers(rng, n, bits, 0)
    nn[:] = 0
    nn[:, bits // 32 - 1] = 0x80000000
    nn[:, bits // 32] = np.uint32(11)                     # 2048 = 2^11
    nn[:, bits // 32 + 1] = 1
    d2, _ = eng.run(bits, api.Operation.add, diag, nn)
    A[np.arange(n) * (n + 1)] = d2
    L = np.zeros_like(A)
    info = la.cholesky(bits, A, n, L)
    Bm = uniform(n * nrhs)
    X = np.zeros_like(Bm)
    ts = la.cholesky_solve(bits, L, n, Bm, nrhs, X)
    # residual R = RN(B - A X) with one rounding per entry (exact GEMM), norms from the rounded values
    R = Bm.copy()
    la.gemm(bits, False, A, X, n, nrhs, n, R, subtract=True)

    def fro(x):
        e = nb.exponent(x).astype(np.float64)
        top = x[:, bits // 32 - 1].astype(np.float64) / 2.0 ** 31
        v = np.where(nb.sign(x) != 0, top * np.exp2(e - np.max(e)), 0.0)
        return np.sqrt(np.sum(v * v)) * 2.0 ** float(np.max(e))
    scaled = fro(R) / (fro(A) * fro(X))
    # the whole factor and the whole solution against the oracle (the reference's blocked sequence, OpenMP)
    orc = Oracle()
    t0 = time.perf_counter()
    WL, winfo = orc.cholesky(bits, A, n, 32)
    t_orc = time.perf_counter() - t0
    factor_match = bool((L == WL).all() and winfo == (info.pivot, info.pivot_sign, info.pivot_status))
    t0 = time.perf_counter()
    WX = orc.solve(bits, WL, n, Bm, nrhs, 32, 3)
    t_orc_solve = time.perf_counter() - t0
    return {"workload": "256-bit blocked Cholesky n=2048 (block 32) + 64-RHS solve", "syrk_s": t_syrk,
            "factor_full_match": factor_match, "solve_full_match": bool((X == WX).all()),
            "oracle_cholesky_s": t_orc, "oracle_solve_s": t_orc_solve, "oracle_cores": os.cpu_count(),
            "cholesky_s": info.timing.wall_seconds, "cholesky_gpu_s": info.timing.gpu_seconds,
            "panel_s": info.panel_seconds, "update_s": info.update_seconds, "pivot": info.pivot,
            "cholesky_mac_per_s": n ** 3 / 6 / info.timing.wall_seconds,
            "solve_s": ts.wall_seconds, "solve_mac_per_s": n * n * nrhs / ts.wall_seconds,
            "scaled_residual": scaled}


def qr_2000(torch, api, scale=1.0):
    """Householder QR least squares on a QSC-like J (m = 2n = 2000, 256 bits, block 32, 4 right-hand sides): column
    scales 2^[-60, 60], entries within 2^-25..2^5 of them, 25% zeros, one entry 2^-150 below the scale in every 17th
    column.  Factor + solve through the host-array API (uploads and downloads included), best of 3; the whole factor
    and solution against the oracle on a scaled copy of the same distribution (m = 400, n = 200 by default)."""
    from limbforge_b200 import numbers as nb
    from oracle.oracle import Oracle
    from tests import qr_cases as qc
    bits, nrhs = 256, 4
    n = max(8, int(round(1000 * scale)))
    m = 2 * n
    rng = np.random.default_rng(31)
    A = qc.matrix(bits, m, n, "qsc", rng)
    B = qc.rhs(bits, m, nrhs, rng)
    eng = api.Engine()
    la = api.Linalg(eng)
    o = api.QROptions(block=32)
    best = None
    for _ in range(3):
        t0 = time.perf_counter()
        qr = la.factor_qr(bits, A, m, n, o)
        t1 = time.perf_counter()
        X = qr.solve(B, nrhs)
        t2 = time.perf_counter()
        run = {"factor_s": t1 - t0, "solve_s": t2 - t1, "e2e_s": t2 - t0, "factor_gpu_s": qr.info.timing.gpu_seconds,
               "panel_s": qr.info.panel_seconds, "update_s": qr.info.update_seconds, "solve_gpu_s": qr.last_timing.gpu_seconds}
        if best is None or run["e2e_s"] < best["e2e_s"]:
            best = run
    # parity: the whole factor and solution of a smaller matrix of the same kind against the oracle
    orc = Oracle()
    ps = int(os.environ.get("LF_QR_PARITY_N", "200"))
    rngp = np.random.default_rng(32)
    Ap = qc.matrix(bits, 2 * ps, ps, "qsc", rngp)
    Bp = qc.rhs(bits, 2 * ps, nrhs, rngp)
    t0 = time.perf_counter()
    want = orc.qr(bits, Ap, 2 * ps, ps, 32)
    t_orc = time.perf_counter() - t0
    got = la.factor_qr(bits, Ap, 2 * ps, ps, o)
    match = all((a == b).all() for a, b in ((got.r(), want["R"]), (got.v(), want["V"]), (got.tau(), want["tau"]), (got.t(), want["T"])))
    match = match and (got.info.rank, got.info.reason, got.info.status) == (want["rank"], want["reason"], want["status"])
    solve_match = bool((got.solve(Bp, nrhs) == orc.qr_solve(want, Bp, nrhs)).all())
    # full-size property: the least-squares residual r = B - A X is orthogonal to the columns of A (A^T r ~ 0)
    Rm = B.copy()
    la.gemm(bits, False, A, X, m, nrhs, n, Rm, subtract=True)
    G = np.zeros((n * nrhs, bits // 32 + 3), np.uint32)
    la.gemm(bits, True, A, Rm, n, nrhs, m, G)

    def mag(x):
        e = nb.exponent(x).astype(np.float64)
        return np.where(nb.sign(x) != 0, e, -np.inf)
    ortho_binades = float(np.max(mag(G)) - (np.max(mag(A)) + np.max(mag(Rm))))
    macs = 2 * m * n * n - 2 * n ** 3 / 3
    return {"workload": f"256-bit Householder QR least squares, QSC-like J {m}x{n} (block 32), {nrhs} right-hand sides",
            **best, "factor_mac_per_s": macs / best["factor_s"], "rank": qr.info.rank, "blocks": qr.info.blocks,
            "reference_m5max_e2e_ms": 529.19 if n == 1000 else None,
            "parity": {"size": f"{2 * ps}x{ps}", "factor_match": bool(match), "solve_match": solve_match, "oracle_s": t_orc},
            "normal_equations_residual_binades": ortho_binades}


def qr_complex_800(torch, api, scale=1.0):
    """Complex Householder QR least squares (256 bits, block 32, 4 right-hand sides) on an 800 x 400 complex QSC-like J
    (real and imaginary parts drawn as the real QR workload's), the shape of the reference's complex QR benchmark; factor +
    solve through the host-array API, best of 3; the whole factor and solution of a 160 x 80 matrix of the same kind
    against the oracle."""
    from oracle.oracle import Oracle
    from tests import qr_cases as qc
    bits, nrhs = 256, 4
    n = max(8, int(round(400 * scale)))
    m = 2 * n
    rng = np.random.default_rng(43)
    A = qc.complex_matrix(bits, m, n, "qsc", rng)
    B = qc.complex_rhs(bits, m, nrhs, rng)
    eng = api.Engine()
    la = api.Linalg(eng)
    o = api.QROptions(block=32)
    best = None
    for _ in range(3):
        t0 = time.perf_counter()
        qr = la.factor_qr_complex(bits, A, m, n, o)
        t1 = time.perf_counter()
        qr.solve(B, nrhs)
        t2 = time.perf_counter()
        run = {"factor_s": t1 - t0, "solve_s": t2 - t1, "e2e_s": t2 - t0, "factor_gpu_s": qr.info.timing.gpu_seconds,
               "panel_s": qr.info.panel_seconds, "update_s": qr.info.update_seconds}
        if best is None or run["e2e_s"] < best["e2e_s"]:
            best = run
    orc = Oracle()
    ps = int(os.environ.get("LF_CQR_PARITY_N", "80"))
    rngp = np.random.default_rng(44)
    Ap = qc.complex_matrix(bits, 2 * ps, ps, "qsc", rngp)
    Bp = qc.complex_rhs(bits, 2 * ps, nrhs, rngp)
    t0 = time.perf_counter()
    want = orc.qr_complex(bits, Ap, 2 * ps, ps, 32)
    t_orc = time.perf_counter() - t0
    got = la.factor_qr_complex(bits, Ap, 2 * ps, ps, o)
    match = all((a == b).all() for a, b in ((got.r(), want["R"]), (got.v(), want["V"]), (got.tau(), want["tau"]), (got.t(), want["T"])))
    match = match and (got.info.rank, got.info.reason, got.info.status) == (want["rank"], want["reason"], want["status"])
    solve_match = bool((got.solve(Bp, nrhs) == orc.qr_complex_solve(want, Bp, nrhs)).all())
    return {"workload": f"256-bit complex Householder QR least squares, QSC-like J {m}x{n} (block 32), {nrhs} right-hand sides",
            **best, "rank": qr.info.rank, "reference_m5max_e2e_ms": 259.28 if n == 400 else None,
            "parity": {"size": f"{2 * ps}x{ps}", "factor_match": bool(match), "solve_match": solve_match, "oracle_s": t_orc}}


def exact_gemm4_448(torch, api, scale=1.0):
    """Exact batched 4 x 4 product, 448-bit complex, 100,000 matrices (the largest configuration of the reference's
    exact 4 x 4 experiment), accumulate into C: resident batch (device time and wall) and host arrays (wall, transfers
    included), beside the composed (rounded-per-step) strided GEMM of the same shape; best of 5 each.  Every result of
    the first 10,000 matrices against the oracle."""
    from limbforge_b200 import numbers as nb
    from oracle.oracle import Oracle
    bits, cx = 448, True
    count = max(16, int(round(100000 * scale)))
    rng = np.random.default_rng(77)
    A, B, C0 = (nb.random_complex(rng, count * 16, bits, 30, zero_frac=0.01, sparse_frac=0.05) for _ in range(3))
    eng = api.Engine()
    g = api.ExactGemm4(eng)
    shape = api.ExactGemm4Shape(count, 16, 16, 16, True, False)
    bufs = [eng.make_buffer(count * 16, bits, cx) for _ in range(3)]
    for b, x in zip(bufs, (A, B, C0)):
        b.upload(x)

    def resident():
        bt = eng.batch()
        g.encode(bt, shape, *bufs)
        return bt.submit().wait()
    for _ in range(3):
        resident()
    res = [resident() for _ in range(5)]
    host = []
    for _ in range(3 + 5):
        C = C0.copy()
        t0 = time.perf_counter()
        g.gemm(bits, cx, shape, A, B, C)
        host.append(time.perf_counter() - t0)
    host = host[3:]
    bl = api.BatchedLinalg(eng)
    sg = api.StridedGemm(count, 4, 4, 4, 16, 16, 16, accumulate=True)
    composed = []
    for _ in range(3 + 5):
        bt = eng.batch()
        bl.gemm_resident(bt, sg, *bufs)
        composed.append(bt.submit().wait())
    composed = composed[3:]
    pc = min(count, 10000)
    sh = {"count": pc, "stride_a": 16, "stride_b": 16, "stride_c": 16, "accumulate": True, "negative": False}
    t0 = time.perf_counter()
    want = Oracle().exact_gemm4(bits, cx, sh, A[:pc * 16], B[:pc * 16], C0[:pc * 16])
    t_orc = time.perf_counter() - t0
    match = bool((C[:pc * 16] == want).all())
    dev_ms = min(t.gpu_seconds for t in res) * 1e3
    # algorithmic bytes: A, B read and C read + written once, 2 * (N + 3) words per complex element
    el = 2 * (bits // 32 + 3) * 4
    moved = count * 16 * el * 4
    return {"workload": f"exact batched 4x4 product, {bits}-bit complex, {count} matrices, accumulate",
            "resident_device_ms": dev_ms, "resident_wall_ms": min(t.wall_seconds for t in res) * 1e3,
            "host_wall_ms": min(host) * 1e3, "composed_device_ms": min(t.gpu_seconds for t in composed) * 1e3,
            "matrices_per_s": count / (dev_ms * 1e-3), "algorithmic_gb_s": moved / (dev_ms * 1e-3) / 1e9,
            "reference_m5max_resident_ms": 49.015 if count == 100000 else None,
            "reference_m5max_host_ms": 49.277 if count == 100000 else None,
            "parity": {"checked_matrices": pc, "match": match},
            "cpu_oracle": {"matrices_per_s": pc / t_orc, "cores": os.cpu_count(), "kind": "port",
                           "sample": f"{pc} of {count} matrices (the C oracle, OpenMP)"}}


def mpfr_bridge():
    """MPFR bridge throughput (host): ns per value of from_mpfr / to_mpfr arrays on one thread and on every host
    thread, beside the mpz route, at 224/256/384/1024 bits and MPFR precisions bits, bits + 64 and bits - 32 (the grid
    of the reference's benchmarks/bridge.cpp), 65,536 values, median of 5.  Built here with g++ against the installed
    MPFR/GMP runtime libraries."""
    import subprocess
    import tempfile
    root = os.path.dirname(os.path.abspath(__file__))
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "bridge")
        subprocess.run(["g++", "-std=c++17", "-O2", f"-I{root}/include", f"-I{root}/tests/cpp/mpfr_decl",
                        os.path.join(root, "tests", "cpp", "bridge.cpp"), "-o", exe, "-l:libmpfr.so.6", "-l:libgmp.so.10",
                        "-pthread"], check=True, capture_output=True)
        ok = subprocess.run([exe, "self"], capture_output=True, text=True, timeout=300)
        r = subprocess.run([exe, "time", "65536", "5"], capture_output=True, text=True, timeout=600, check=True)
    rows = [json.loads(line) for line in r.stdout.splitlines() if line.startswith("{")]
    return {"workload": "MPFR bridge, 65,536 values per array", "self_checks": "bridge ok" in ok.stdout, "rows": rows,
            "reference_m5max": "2-4 ns/value for threaded arrays on 3-16 threads (docs/optimizations.md, loaded host)"}


def ragged_batch(torch, api, scale=1.0):
    """20,000 complex GEMMs, m, n, k uniform in {4..48}, precision uniform in {128, 256, 512, 1024},
    plus 200,000 4x4 complex LU solves at 512 bits, as one CUDA graph launch of a tuned ragged plan
    (`scale` shrinks both counts, for profiling captures)."""
    from limbforge_b200 import numbers as nb
    from oracle.oracle import Oracle
    rng = np.random.default_rng(104)
    count, lu_count = max(16, int(20000 * scale)), max(64, int(200000 * scale))
    bits = rng.choice([128, 256, 512, 1024], size=count)
    m, n, k = (rng.integers(4, 49, size=count) for _ in range(3))
    items = api.ragged_items(bits, m, n, k)
    lu = api.RaggedLu4(512, api.Batched4(count=lu_count, rhs=1))
    total = api.ragged_pack(True, items, lu)
    arena = np.zeros(total // 4, np.uint32)
    for it in items:
        b, mm, nn, kk = int(it["bits"]), int(it["m"]), int(it["n"]), int(it["k"])
        x = nb.random_complex(rng, mm * kk + kk * nn, b, 32)
        w = x.shape[1] * x.shape[2]
        a0, b0 = int(it["a"]) // 4, int(it["b"]) // 4
        arena[a0:a0 + mm * kk * w] = x[:mm * kk].ravel()
        arena[b0:b0 + kk * nn * w] = x[mm * kk:].ravel()
    LA = nb.random_complex(rng, lu_count * 16, 512, 32).ravel()
    LB = nb.random_complex(rng, lu_count * 4, 512, 32).ravel()
    arena[lu.A // 4:lu.A // 4 + LA.size] = LA
    arena[lu.B // 4:lu.B // 4 + LB.size] = LB
    eng = api.Engine()
    plan = api.RaggedPlan(eng, True, False, items, total, lu)
    dev = torch.from_numpy(arena.view(np.int32)).cuda()
    ptr = dev.data_ptr()
    t0 = time.perf_counter()
    plan.tune(ptr)
    t_tune = time.perf_counter() - t0
    st = torch.cuda.current_stream()
    for _ in range(2):
        plan.run(ptr, st.cuda_stream)
    ms = _event_ms(torch, st, lambda: plan.run(ptr, st.cuda_stream), 5)
    out = dev.cpu().numpy().view(np.uint32)
    # the oracle on 1,000 instances (every class, k up to 48) and on every LU system, on all host cores
    from concurrent.futures import ThreadPoolExecutor
    orc = Oracle()
    sample = rng.choice(count, size=min(count, 1000), replace=False)

    def instance_ok(t):
        it = items[t]
        b, mm, nn, kk = int(it["bits"]), int(it["m"]), int(it["n"]), int(it["k"])
        w = 2 * (b // 32 + 3)
        Am = arena[int(it["a"]) // 4:int(it["a"]) // 4 + mm * kk * w].reshape(-1, 2, w // 2)
        Bm = arena[int(it["b"]) // 4:int(it["b"]) // 4 + kk * nn * w].reshape(-1, 2, w // 2)
        want = orc.strided_gemm(b, True, {"count": 1, "m": mm, "n": nn, "k": kk, "stride_a": 0, "stride_b": 0, "stride_c": 0},
                                np.ascontiguousarray(Am), np.ascontiguousarray(Bm), np.zeros((mm * nn, 2, w // 2), np.uint32))
        return bool((out[int(it["c"]) // 4:int(it["c"]) // 4 + want.size] == want.ravel()).all())
    t0 = time.perf_counter()
    with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        oks = list(ex.map(instance_ok, sample))
    Aall = np.ascontiguousarray(arena[lu.A // 4:lu.A // 4 + LA.size].reshape(lu_count * 16, 2, 19))
    Ball = np.ascontiguousarray(arena[lu.B // 4:lu.B // 4 + LB.size].reshape(lu_count * 4, 2, 19))
    X, _, stt = orc.lu4(512, lu_count, 1, 0, Aall, Ball)
    t_orc = time.perf_counter() - t0
    Xg = out[lu.X // 4:lu.X // 4 + lu_count * 4 * 38]
    Sg = out[lu.status // 4:lu.status // 4 + lu_count]
    lu_ok = bool((Xg == X.ravel()).all() and (Sg == stt).all())
    # the LU job alone: a plan holding only the 200,000 systems, on the same device data
    lu_alone = api.RaggedPlan(eng, True, False, api.ragged_items([], [], [], []), total, lu)
    lu_alone.tune(ptr)
    for _ in range(2):
        lu_alone.run(ptr, st.cuda_stream)
    lu_ms = _event_ms(torch, st, lambda: lu_alone.run(ptr, st.cuda_stream), 5)
    word_macs = float(np.sum(m.astype(np.float64) * n * k * 4 * (bits // 32) ** 2))
    return {"workload": f"{count} ragged complex GEMMs (m,n,k U{{4..48}}, bits U{{128,256,512,1024}}) + {lu_count} 4x4 LU at 512 bits, one graph launch",
            "graph_ms": ms, "instances_per_s": count / (ms * 1e-3),
            "lu4_alone_ms": lu_ms, "lu4_systems_per_s_alone": lu_count / (lu_ms * 1e-3), "lu4_plan": lu_alone.info(),
            "gemm_word_macs_per_s": word_macs / (ms * 1e-3), "complex_macs": float(np.sum(m.astype(np.float64) * n * k)),
            "arena_bytes": int(total), "tune_s": t_tune, "plan": plan.info(),
            "instances_checked": int(len(sample)), "instances_full_match": bool(all(oks)), "instance_mismatches": int(len(oks) - sum(oks)),
            "lu4_checked": lu_count, "lu4_full_match": lu_ok, "oracle_s": t_orc}


def run_workloads(args):
    import torch
    from limbforge_b200 import api
    hbm_peak, _ = peaks()
    out = {}
    for name, fn in (("mul_div_fma_256bit_65536", lambda: elementwise_256(torch, api, hbm_peak)),
                     ("cdiv_1024bit_65536", lambda: cdiv_1024(torch, api)),
                     ("exact_gemm_512bit_1024", lambda: exact_gemm_512(torch, api, args.scale)),
                     ("cholesky_256bit_2048", lambda: cholesky_2048(torch, api)),
                     ("qr_256bit_2000x1000", lambda: qr_2000(torch, api, args.scale)),
                     ("qr_complex_256bit_800x400", lambda: qr_complex_800(torch, api, args.scale)),
                     ("exact_gemm4_448bit_complex_100000", lambda: exact_gemm4_448(torch, api, args.scale)),
                     ("ragged_batch_20000", lambda: ragged_batch(torch, api, args.scale)),
                     ("mpfr_bridge", mpfr_bridge)):
        if args.workload and name != args.workload:
            continue
        t0 = time.perf_counter()
        try:
            out[name] = fn()
        except Exception as e:                       # reported, never hidden
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        _log(f"{name} done in {time.perf_counter() - t0:.1f} s")
        torch.cuda.empty_cache()
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    from limbforge_b200 import api, shard

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist_
        dist = dist_
    x, f = make_inputs(20261203 + rank)
    E = BITS // 32 + 3
    # device-resident inputs (torch only as the allocator and stream owner)
    dx = torch.from_numpy(x.view(np.int32)).cuda()
    df = torch.from_numpy(np.ascontiguousarray(f).view(np.int32)).cuda()
    dout = torch.empty_like(dx)
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream

    def step():
        api.dev_mul_chain(BITS, dx.data_ptr(), df.data_ptr(), COUNT, CHAIN, dout.data_ptr(), COUNT, stream=sp)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()
    # correctness of the timed kernel on this rank's data: a sample against the oracle
    got = dout.cpu().numpy().view(np.uint32)
    chain_full_match = None
    if rank == 0:
        from oracle.oracle import Oracle
        want = Oracle().mul_chain(BITS, x, np.ascontiguousarray(f))
        chain_full_match = bool((got == want).all())
        assert chain_full_match, "chain result differs from the oracle"

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for _ in range(args.steps):
                step()
            ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    # A/B of the warp-cooperative form: one value per lane pair (same bits), timed the same way on rank 0's data
    lanes_ab = None
    if world == 1:
        dpair = torch.empty_like(dx)

        def pair_step():
            api.dev_mul_chain_lanes(BITS, 2, dx.data_ptr(), df.data_ptr(), COUNT, CHAIN, dpair.data_ptr(), COUNT, stream=sp)
        with torch.cuda.stream(stream):
            for _ in range(max(3, args.warmup)):
                pair_step()
        torch.cuda.synchronize()
        pair_same = bool(torch.equal(dpair, dout))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(args.steps):
                pair_step()
            e1.record(stream)
        torch.cuda.synchronize()
        lanes_ab = {"one_value_per_thread_ms": ms / args.steps, "one_value_per_lane_pair_ms": e0.elapsed_time(e1) / args.steps,
                    "lane_pair_bits_identical": pair_same}
        del dpair
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms_total = shard.max_over_ranks(ms, dist, "cuda")            # the job's time is its slowest rank's
    ms_step = ms_total / args.steps
    value = world * COUNT * CHAIN / (ms_step * 1e-3)

    # ---- end to end through the public API with pinned host buffers
    hx = api.PinnedArray(x.shape)
    hf = api.PinnedArray(f.shape)
    ho = api.PinnedArray(x.shape)
    hx.array[...] = x
    hf.array[...] = f
    eng = api.Engine(device=local_rank)
    X = eng.make_buffer(COUNT, BITS)
    F = [eng.make_buffer(COUNT, BITS) for _ in range(CHAIN)]

    def e2e_step():
        X.upload(hx.array)
        for s in range(CHAIN):
            F[s].upload(hf.array[s])
        b = eng.batch()
        for s in range(CHAIN):
            b.run(api.Operation.mul, X, F[s], None, X)
        b.submit().wait()
        X.download(out=ho.array)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    assert (ho.array == got).all(), "public-API chain differs from the device entry point"
    e2e_steps = max(3, min(args.steps, 20))
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_s = shard.max_over_ranks((time.perf_counter() - t0) / e2e_steps, dist, "cuda")
    e2e_value = world * COUNT * CHAIN / e2e_s

    if rank != 0:
        return
    hbm_peak, peak_kind = peaks()
    bytes_per_launch = COUNT * (CHAIN + 2) * ELEMENT_BYTES          # x, 16 factors read; result written
    achieved = bytes_per_launch / (ms_step * 1e-3) / 1e9
    word_macs = COUNT * CHAIN * (BITS // 32) ** 2
    sample = int(os.environ.get("LF_CPU_SAMPLE", "8192"))
    cpu_rate, kind, cores = cpu_reference_rate(x, f, sample)
    mpfr = mpfr_chain_rates(x, f, got)
    peak_macs = word_mac_peak(api, local_rank)
    executed = COUNT * CHAIN * UPPER_PRODUCTS
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32 limbs (1024-bit RNE)", "data": "synthetic",
        "config": {"workload": WORKLOAD, "count": COUNT, "steps_per_chain": CHAIN, "bits": BITS,
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "l2": "inputs larger than L2 (%.0f MB resident per step)" % (bytes_per_launch / 1e6)},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(x.nbytes + f.nbytes),
                "d2h_bytes_per_step": int(x.nbytes), "ms_per_step": e2e_s * 1e3},
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                     "traffic": TRAFFIC_BYTES, "peak_kind": peak_kind,
                     "note": "the 1024-bit chain kernel is integer-pipe bound; HBM fraction shown per the contract"},
        "integer_pipe": {
            "bound": "integer multiply-add pipe", "unit": "word-MAC/s",
            "algorithmic_word_macs_per_step": word_macs, "algorithmic_word_macs_per_s": word_macs / (ms_step * 1e-3),
            "executed_word_macs_per_step": executed, "executed_word_macs_per_s": executed / (ms_step * 1e-3),
            "peak": peak_macs, "peak_kind": "measured: lf_probe_word_mac_rate, 8 independent 32x32->64 multiply-add chains per thread",
            "frac": (executed / (ms_step * 1e-3) / peak_macs) if peak_macs else None,
            "note": "executed counts the upper-half product's 559 word products per 1024-bit product (algorithmic: 1024)"},
        "clocks": clocks.summary(),
        "cpu_baseline": {"value": cpu_rate, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{sample} of {COUNT} values x {CHAIN} steps, extrapolated",
                         "mpfr": mpfr},
        "chain_full_match": chain_full_match,
        "chain_lanes_ab": lanes_ab,
    }
    if mpfr.get("all_core_ops_per_s"):
        line["vs_mpfr_all_core"] = {"value": value / mpfr["all_core_ops_per_s"], "e2e": e2e_value / mpfr["all_core_ops_per_s"],
                                    "serial_value": value / mpfr["serial_ops_per_s"]}
    if world == 1 and not args.no_workloads:
        line["workloads"] = run_workloads(args)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--count", type=int, default=65536, help="values per chain (65,536 is the headline workload)")
    ap.add_argument("--no-workloads", action="store_true", help="skip the secondary workloads")
    ap.add_argument("--workload", default="", help="run only this secondary workload and print its JSON (profiling)")
    ap.add_argument("--scale", type=float, default=1.0, help="size factor of the ragged batch and the exact GEMM (profiling captures)")
    args = ap.parse_args()
    global COUNT
    COUNT = args.count
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload:
        import torch
        torch.cuda.set_device(local_rank)
        print(json.dumps(run_workloads(args)), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
