"""GPU: ragged mixed-precision batches (lf_ragged_plan_*) against the C oracle, bit for bit.

Each instance must equal a one-instance StridedGemm at its own precision as the oracle computes it
(ascending k, composed or fused complex updates, accumulate and negate per instance), the LU job
must equal the oracle's batched 4x4 solve, inputs must stay untouched, and the autotuner's trial runs
must not change the arena.  Shapes include empty instances (m, n or k zero) and every precision class
in one plan; validation rejects overlapping outputs, outputs over inputs, misaligned offsets and
operands outside the arena."""
import numpy as np
import pytest

from limbforge_b200 import api
from limbforge_b200 import numbers as nb

pytestmark = pytest.mark.gpu


def make_case(rng, count, bits_choices, max_dim, complex_=True, lu_count=0, zero_dims=True, min_dim=None):
    bits = rng.choice(bits_choices, size=count)
    lo = (0 if zero_dims else 1) if min_dim is None else min_dim
    m, n, k = (rng.integers(lo, max_dim + 1, size=count) for _ in range(3))
    acc = rng.integers(0, 2, size=count)
    neg = rng.integers(0, 2, size=count)
    items = api.ragged_items(bits, m, n, k, acc, neg)
    lu = api.RaggedLu4(512, api.Batched4(count=lu_count, rhs=1, determinant=True)) if lu_count else None
    total = api.ragged_pack(complex_, items, lu)
    arena = np.zeros(total // 4, np.uint32)

    def rand(b, cnt):
        return nb.random_complex(rng, cnt, b, 32) if complex_ else nb.random_numbers(rng, cnt, b, 32)

    for it in items:
        b = int(it["bits"])
        for off, cnt in ((it["a"], it["m"] * it["k"]), (it["b"], it["k"] * it["n"]), (it["c"], it["m"] * it["n"])):
            if cnt:
                x = rand(b, int(cnt)).ravel()
                arena[int(off) // 4:int(off) // 4 + x.size] = x
    if lu:
        A = nb.random_complex(rng, lu_count * 16, 512, 32).ravel()
        B = nb.random_complex(rng, lu_count * 4, 512, 32).ravel()
        arena[lu.A // 4:lu.A // 4 + A.size] = A
        arena[lu.B // 4:lu.B // 4 + B.size] = B
    return items, lu, arena


def view(arena, off, cnt, bits, complex_):
    w = nb.element_words(bits) * (2 if complex_ else 1)
    x = arena[int(off) // 4:int(off) // 4 + int(cnt) * w]
    return x.reshape(int(cnt), 2, w // 2) if complex_ else x.reshape(int(cnt), w)


def expected(oracle, items, lu, arena, complex_, fused):
    out = arena.copy()
    for it in items:
        b, m, n, k = int(it["bits"]), int(it["m"]), int(it["n"]), int(it["k"])
        if not m * n:
            continue
        A = view(arena, it["a"], max(m * k, 1), b, complex_) if k else np.zeros((1, 2, nb.element_words(b)) if complex_ else (1, nb.element_words(b)), np.uint32)
        B = view(arena, it["b"], max(k * n, 1), b, complex_) if k else A
        Cm = view(arena, it["c"], m * n, b, complex_)
        s = {"count": 1, "m": m, "n": n, "k": k, "stride_a": m * k, "stride_b": k * n, "stride_c": m * n,
             "accumulate": bool(it["accumulate"]), "fused": fused, "negative": bool(it["negative"])}
        want = oracle.strided_gemm(b, complex_, s, np.ascontiguousarray(A), np.ascontiguousarray(B), np.ascontiguousarray(Cm))
        out[int(it["c"]) // 4:int(it["c"]) // 4 + want.size] = want.ravel()
    if lu:
        c = lu.shape.count
        A = view(arena, lu.A, c * 16, 512, True)
        B = view(arena, lu.B, c * 4, 512, True)
        X, det, st = oracle.lu4(512, c, 1, 2, np.ascontiguousarray(A), np.ascontiguousarray(B))
        out[lu.X // 4:lu.X // 4 + X.size] = X.ravel()
        out[lu.det // 4:lu.det // 4 + det.size] = det.ravel()
        out[lu.status // 4:lu.status // 4 + st.size] = st
    return out


def run_plan(engine, plan, arena, tune=False):
    buf = engine.make_buffer(arena.size)
    buf.upload(arena)
    ptr = buf.device_pointer()
    if tune:
        plan.tune(ptr)
    plan.run(ptr)
    return buf.download()


@pytest.mark.parametrize("fused", [False, True])
def test_ragged_complex_batch_with_lu_vs_oracle(engine, oracle, fused):
    rng = np.random.default_rng(11 + fused)
    items, lu, arena = make_case(rng, 160, [64, 96, 128, 256, 384, 512, 1024], 7, lu_count=96)
    plan = api.RaggedPlan(engine, True, fused, items, arena.size * 4, lu)
    got = run_plan(engine, plan, arena)
    want = expected(oracle, items, lu, arena, True, fused)
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, f"first differing word {bad[:5]}"
    info = plan.info()
    assert {c["bits"] for c in info["classes"]} == {int(b) for b, m, n in zip(items["bits"], items["m"], items["n"]) if m * n}
    assert sum(c["items"] for c in info["classes"]) == int(np.count_nonzero(items["m"] * items["n"]))


@pytest.mark.parametrize("fused", [False, True])
def test_ragged_benchmark_shapes_vs_oracle(engine, oracle, fused):
    """The benchmark's shape distribution: m, n, k uniform in {4..48}, precision uniform over
    {128, 256, 512, 1024} bits, with 1,200 LU systems at 512 bits in the same tuned plan; every output
    word is compared (the 1024-bit class runs its parked-state kernel at k up to 48)."""
    rng = np.random.default_rng(48 + fused)
    items, lu, arena = make_case(rng, 240, [128, 256, 512, 1024], 48, lu_count=1200, min_dim=4)
    plan = api.RaggedPlan(engine, True, fused, items, arena.size * 4, lu)
    got = run_plan(engine, plan, arena, tune=True)
    want = expected(oracle, items, lu, arena, True, fused)
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, f"first differing word {bad[:5]}"
    assert {c["bits"] for c in plan.info()["classes"]} == {128, 256, 512, 1024}


def test_ragged_tuned_equals_untuned_and_arena_is_kept(engine, oracle):
    rng = np.random.default_rng(5)
    items, lu, arena = make_case(rng, 120, [128, 256, 512, 1024], 9, lu_count=200, zero_dims=False)
    plan = api.RaggedPlan(engine, True, False, items, arena.size * 4, lu)
    first = run_plan(engine, plan, arena)
    # the tuner's trial runs write to plan scratch: the arena after tune + run equals one run
    tuned = run_plan(engine, plan, arena, tune=True)
    assert (first == tuned).all()
    info = plan.info()
    assert info["tuned"] and info["lu4_block"] in (32, 64, 128, 256)
    for c in info["classes"]:
        assert c["block"] in (32, 64, 128, 256) and c["grid"] > 0 and c["trial_ms"] > 0
    want = expected(oracle, items, lu, arena, True, False)
    assert (tuned == want).all()


def test_ragged_real_batch_repeated_runs_and_moved_arena(engine, oracle):
    rng = np.random.default_rng(8)
    items, _, arena = make_case(rng, 90, [64, 160, 288, 992], 6, complex_=False)
    items["accumulate"] = 0                      # repeated runs give the same outputs
    plan = api.RaggedPlan(engine, False, True, items, arena.size * 4)
    buf = engine.make_buffer(arena.size)
    buf.upload(arena)
    plan.run(buf.device_pointer())
    plan.run(buf.device_pointer())
    got = buf.download()
    want = expected(oracle, items, None, arena, False, True)
    assert (got == want).all()
    buf2 = engine.make_buffer(arena.size)        # a second arena: the graph is rebuilt for it
    buf2.upload(arena)
    plan.run(buf2.device_pointer())
    assert (buf2.download() == want).all()


def test_ragged_matches_strided_gemm(engine):
    """A ragged plan of equal shapes gives the bits of one StridedGemm call over the same data."""
    rng = np.random.default_rng(21)
    count, m, n, k, bits = 40, 5, 6, 7, 384
    items = api.ragged_items([bits] * count, [m] * count, [n] * count, [k] * count)
    total = api.ragged_pack(True, items)
    A = nb.random_complex(rng, count * m * k, bits, 32)
    B = nb.random_complex(rng, count * k * n, bits, 32)
    C0 = nb.random_complex(rng, count * m * n, bits, 32)
    arena = np.zeros(total // 4, np.uint32)
    for t, it in enumerate(items):
        for off, src, sz in ((it["a"], A, m * k), (it["b"], B, k * n), (it["c"], C0, m * n)):
            x = src[t * sz:(t + 1) * sz].ravel()
            arena[int(off) // 4:int(off) // 4 + x.size] = x
    plan = api.RaggedPlan(engine, True, False, items, total)
    got = run_plan(engine, plan, arena)
    Cs = C0.copy()
    api.BatchedLinalg(engine).gemm(bits, True, api.StridedGemm(count, m, n, k, m * k, k * n, m * n), A, B, Cs)
    for t, it in enumerate(items):
        assert (view(got, it["c"], m * n, bits, True) == Cs[t * m * n:(t + 1) * m * n]).all()


def test_ragged_validation(engine):
    items = api.ragged_items([256, 256], [2, 2], [2, 2], [2, 2])
    total = api.ragged_pack(True, items)
    bad = items.copy()
    bad["c"][1] = bad["c"][0]                    # two outputs on the same bytes
    with pytest.raises(api.InvalidArgument, match="overlap"):
        api.RaggedPlan(engine, True, False, bad, total)
    bad = items.copy()
    bad["c"][1] = bad["a"][0]                    # an output over an input
    with pytest.raises(api.InvalidArgument, match="overlaps an input"):
        api.RaggedPlan(engine, True, False, bad, total)
    bad = items.copy()
    bad["a"][0] += 4
    with pytest.raises(api.InvalidArgument, match="multiples of 16"):
        api.RaggedPlan(engine, True, False, bad, total)
    with pytest.raises(api.InvalidArgument, match="outside the arena"):
        api.RaggedPlan(engine, True, False, items, total - 256)
    empty = api.RaggedPlan(engine, True, False, api.ragged_items([], [], [], []), 0)
    empty.run(0)
