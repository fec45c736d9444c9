"""GPU parity of the element-wise path through the C ABI (host-array calls, resident batches
with chain fusion, device-pointer entry points) against the golden vectors and the C oracle,
bit for bit; plus the reference's ownership and argument errors
(tests/test_arithmetic.cpp, test_fused.cpp, test_broadcast.cpp, test_buffers.cpp)."""
import numpy as np
import pytest

from limbforge_b200 import numbers as nb

pytestmark = pytest.mark.gpu

GOLDEN_WIDTHS = [64, 96, 128, 224, 256, 384, 512, 1024]
ALL_WIDTHS = list(range(64, 1025, 32))


def same(x, y):
    return x.shape == y.shape and bool((x == y).all())


def first_bad(x, y):
    d = np.nonzero((x != y).reshape(x.shape[0], -1).any(axis=1))[0]
    return d[:5]


@pytest.mark.parametrize("bits", GOLDEN_WIDTHS)
def test_golden_real(engine, golden, bits):
    from limbforge_b200.api import Operation
    a, b, roots = golden[f"real_{bits}_a"], golden[f"real_{bits}_b"], golden[f"real_{bits}_roots"]
    for op in (0, 1, 2, 3):
        out, _ = engine.run(bits, Operation(op), a, b)
        want = golden[f"real_{bits}_{op}_out"]
        assert same(out, want), f"op {op} bad cases {first_bad(out, want)}"
    for op, x in ((7, a), (8, roots)):
        out, _ = engine.run_unary(bits, Operation(op), x)
        want = golden[f"real_{bits}_{op}_out"]
        assert same(out, want), f"op {op} bad cases {first_bad(out, want)}"


@pytest.mark.parametrize("bits", GOLDEN_WIDTHS)
def test_golden_fused_and_complex(engine, golden, bits):
    from limbforge_b200.api import Operation
    fa, fb, fc = golden[f"fused_{bits}_a"], golden[f"fused_{bits}_b"], golden[f"fused_{bits}_c"]
    for op in (9, 10):
        out, _ = engine.run_ternary(bits, Operation(op), fa, fb, fc)
        want = golden[f"fused_{bits}_{op}_out"]
        assert same(out, want), f"op {op} bad cases {first_bad(out, want)}"
    ca, cb, cc = golden[f"cx_{bits}_a"], golden[f"cx_{bits}_b"], golden[f"cx_{bits}_c"]
    for op in (4, 5, 6):
        out, _ = engine.run(bits, Operation(op), ca, cb)
        want = golden[f"cx_{bits}_{op}_out"]
        assert same(out, want), f"op {op} bad cases {first_bad(out, want)}"
    for op in (11, 12):
        out, _ = engine.run_ternary(bits, Operation(op), ca, cb, cc)
        want = golden[f"cx_{bits}_{op}_out"]
        assert same(out, want), f"op {op} bad cases {first_bad(out, want)}"


@pytest.mark.parametrize("bits", ALL_WIDTHS)
def test_every_width_vs_oracle(engine, oracle, bits):
    from limbforge_b200.api import Operation
    rng = np.random.default_rng(1000 + bits)
    n = bits // 32
    cnt = 1024
    a = nb.random_numbers(rng, cnt, bits, 1000, zero_frac=0.03, sparse_frac=0.05)
    b = nb.random_numbers(rng, cnt, bits, 1000, zero_frac=0.03, sparse_frac=0.05)
    c = nb.random_numbers(rng, cnt, bits, 1500, zero_frac=0.03, sparse_frac=0.05)
    b[::3, n] = (nb.exponent(a[::3]) - rng.integers(0, bits + 80, size=a[::3].shape[0])).astype(np.int32).view(np.uint32)
    b[1::9] = nb.negate(a[1::9])
    b[1::9, 0] ^= np.uint32(3)
    c[2::7] = nb.negate(oracle.elementwise(bits, 2, a[2::7].copy(), b[2::7].copy()))
    a[5::97, n + 2] = nb.INVALID
    for op in (0, 1, 2, 3, 7):
        out = engine.run(bits, Operation(op), a, b)[0] if op != 7 else engine.run_unary(bits, Operation(op), a)[0]
        want = oracle.elementwise(bits, op, a, b)
        assert same(out, want), f"op {op} bad {first_bad(out, want)}"
    r = a.copy()
    r[:, n + 1] = np.abs(nb.sign(r)).astype(np.int32).view(np.uint32)
    assert same(engine.run_unary(bits, Operation.sqrt, r)[0], oracle.elementwise(bits, 8, r))
    for op in (9, 10):
        out = engine.run_ternary(bits, Operation(op), a, b, c)[0]
        want = oracle.elementwise(bits, op, a, b, c)
        assert same(out, want), f"op {op} bad {first_bad(out, want)}"
    ca, cb, cc = (nb.random_complex(rng, 96, bits, 30) for _ in range(3))
    cb[::5, 0], cb[::5, 1] = ca[::5, 1], ca[::5, 0]
    for op in (4, 5, 6):
        assert same(engine.run(bits, Operation(op), ca, cb)[0], oracle.elementwise(bits, op, ca, cb)), f"complex op {op}"
    for op in (11, 12):
        assert same(engine.run_ternary(bits, Operation(op), ca, cb, cc)[0], oracle.elementwise(bits, op, ca, cb, cc)), f"op {op}"


def boundary_operands(bits, cnt=4096):
    """Operand pairs whose products put runs of zeros or ones around the rounding position, exact
    ties and exact results."""
    n = bits // 32
    rng = np.random.default_rng(bits + 5)
    a = nb.random_numbers(rng, cnt, bits, 50)
    b = nb.random_numbers(rng, cnt, bits, 50)
    q = cnt // 8
    # a = 2^(32n-1) + u: the product is b shifted plus a small multiple of b
    a[:q, :n] = 0
    a[:q, n - 1] = 0x80000000
    a[:q, 0] = rng.integers(0, 1 << 20, size=q)
    # trailing words of all zeros / all ones in both operands
    a[q:2 * q, :n // 2] = 0
    b[q:2 * q, :n // 2] = 0
    a[2 * q:3 * q, :n - 1] = 0xFFFFFFFF
    b[2 * q:3 * q, :n - 1] = 0xFFFFFFFF
    # b = 2^(32n-1) + 2^(32n-2): exact products 1.5 x a, ties when a is odd
    b[3 * q:4 * q, :n] = 0
    b[3 * q:4 * q, n - 1] = 0xC0000000
    # one limb set below the top, at every position
    b[4 * q:5 * q, :n - 1] = 0
    b[4 * q + np.arange(q), np.arange(q) % (n - 1)] = rng.integers(1, 1 << 32, size=q, dtype=np.uint64).astype(np.uint32)
    # squares of numbers close to a power of two (products just below / above 2^(64n-2))
    a[5 * q:6 * q, :n] = 0xFFFFFFFF
    a[5 * q:6 * q, 0] = rng.integers(0, 1 << 32, size=q, dtype=np.uint64).astype(np.uint32)
    b[5 * q:6 * q] = a[5 * q:6 * q]
    return a, b


@pytest.mark.parametrize("bits", [256, 384, 512, 800, 1024])
def test_mul_near_rounding_boundaries(engine, oracle, bits):
    """From 12 limbs on, mul decides the rounding from the upper part of the product and must fall
    back to the full product exactly in the boundary cases."""
    from limbforge_b200.api import Operation
    a, b = boundary_operands(bits)
    out, _ = engine.run(bits, Operation.mul, a, b)
    want = oracle.elementwise(bits, 2, a, b)
    assert same(out, want), f"first differing element {first_bad(out, want)}"


@pytest.mark.parametrize("bits", [384, 512, 800, 1024])
def test_chain_mul_near_rounding_boundaries(oracle, bits):
    """The chain kernel's product reads the factor's words from memory inside the product; the same
    boundary operands through a one-step chain give the oracle's products."""
    from limbforge_b200 import api
    a, b = boundary_operands(bits)
    count = a.shape[0]
    e = api.Engine()
    X, F, O = e.make_buffer(count, bits), e.make_buffer(count, bits), e.make_buffer(count, bits)
    X.upload(a)
    F.upload(b)
    api.dev_mul_chain(bits, X.device_pointer(), F.device_pointer(), count, 1, O.device_pointer(), count)
    assert same(O.download(), oracle.elementwise(bits, 2, a, b))


@pytest.mark.parametrize("bits", [384, 448, 512, 640, 832, 1024])
def test_chain_on_lane_pairs(oracle, bits):
    """Chains with one value per lane pair (lf_dev_mul_chain_lanes, lanes = 2): the boundary operands through a
    one-step chain, and a 9-step chain over a count that leaves a partial block, give the oracle's bits."""
    from limbforge_b200 import api
    a, b = boundary_operands(bits)
    count = a.shape[0]
    e = api.Engine()
    X, F, O = e.make_buffer(count, bits), e.make_buffer(count, bits), e.make_buffer(count, bits)
    X.upload(a)
    F.upload(b)
    api.dev_mul_chain_lanes(bits, 2, X.device_pointer(), F.device_pointer(), count, 1, O.device_pointer(), count)
    assert same(O.download(), oracle.elementwise(bits, 2, a, b))
    rng = np.random.default_rng(bits + 9)
    count, steps = 1000 + 17, 9
    x = nb.random_numbers(rng, count, bits, 8, zero_frac=0.01, sparse_frac=0.02)
    f = np.stack([nb.random_numbers(rng, count, bits, 8, zero_frac=0.01, sparse_frac=0.02) for _ in range(steps)])
    X, F, O = e.make_buffer(count, bits), e.make_buffer(count * steps, bits), e.make_buffer(count, bits)
    X.upload(x)
    F.upload(f.reshape(count * steps, -1))
    api.dev_mul_chain_lanes(bits, 2, X.device_pointer(), F.device_pointer(), count, steps, O.device_pointer(), count)
    assert same(O.download(), oracle.mul_chain(bits, x, f))


def test_chain_factor_written_earlier_in_the_chain(engine, oracle):
    """y1 = x * f, y2 = y1 * y1, y3 = y2 * f: the second step's factor is the first step's output,
    written earlier in the same fused kernel."""
    from limbforge_b200.api import Operation
    bits, count = 1024, 2048
    rng = np.random.default_rng(12)
    x, f = nb.random_numbers(rng, count, bits, 6), nb.random_numbers(rng, count, bits, 6)
    X, F = engine.make_buffer(count, bits), engine.make_buffer(count, bits)
    Y1, Y2, Y3 = (engine.make_buffer(count, bits) for _ in range(3))
    X.upload(x)
    F.upload(f)
    batch = engine.batch()
    batch.run(Operation.mul, X, F, None, Y1)
    batch.run(Operation.mul, Y1, Y1, None, Y2)
    batch.run(Operation.mul, Y2, F, None, Y3)
    batch.submit().wait()
    y1 = oracle.elementwise(bits, 2, x, f)
    y2 = oracle.elementwise(bits, 2, y1, y1)
    assert same(Y1.download(), y1)
    assert same(Y2.download(), y2)
    assert same(Y3.download(), oracle.elementwise(bits, 2, y2, f))


def sqrt_operands(bits, cnt=2048):
    """Positive radicands for sqrt: random values of both exponent parities, exact squares, roots just
    below and just above a half unit (the rounding boundary), and the ends of the binade."""
    n = bits // 32
    rng = np.random.default_rng(bits + 77)
    x = nb.random_numbers(rng, cnt, bits, 60)
    x[:, n + 1] = 1
    q = cnt // 8

    def put(row, m, odd):
        for w in range(n):
            x[row, w] = (m >> (32 * w)) & 0xFFFFFFFF
        x[row, n] = np.int32(2 * int(rng.integers(-20, 21)) + odd).view(np.uint32)

    # the radicand is Z = m 2^(32n) for an odd exponent, m 2^(32n-1) for an even one
    for t in range(q):                                     # exact squares
        r = (int(rng.integers(1 << 30, 1 << 31)) << (32 * n - 31)) >> (16 * n) << (16 * n)
        r |= 1 << (32 * n - 1)
        z = r * r
        if z >> (64 * n - 1):
            put(t, z >> (32 * n), 1)
        else:
            put(t, z >> (32 * n - 1), 0)
    for t in range(q, 3 * q):                              # sqrt(Z) within a hair of k + 1/2
        k = int.from_bytes(rng.bytes(4 * n), "little") | (1 << (32 * n - 1))
        z = k * k + k                                      # (k + 1/2)^2 - 1/4
        odd = 1 if z >> (64 * n - 1) else 0
        sh = 32 * n if odd else 32 * n - 1
        put(t, (z >> sh) + (t & 1), odd)
    for t in range(3 * q, 4 * q):                          # binade ends: 2^(32n-1) and 2^(32n) - 1
        put(t, (1 << (32 * n - 1)) if t & 2 else (1 << (32 * n)) - 1, t & 1)
    return x


@pytest.mark.parametrize("bits", list(range(64, 1025, 32)))
def test_sqrt_all_widths_and_hard_cases(engine, oracle, bits):
    """sqrt's candidate comes from a fixed-point reciprocal square root and one exact correction; the
    exact check must then land on the oracle's correctly rounded root at every width."""
    from limbforge_b200.api import Operation
    x = sqrt_operands(bits)
    out, _ = engine.run_unary(bits, Operation.sqrt, x)
    want = oracle.elementwise(bits, 8, x)
    assert same(out, want), f"first differing element {first_bad(out, want)}"


@pytest.mark.parametrize("bits", [64, 224, 256, 384, 1024])
def test_broadcast_operands(engine, oracle, bits):
    """tests/test_broadcast.cpp: b (and c) read at (i / stride) % period."""
    from limbforge_b200.api import Broadcast, Operation, broadcast_elements
    rng = np.random.default_rng(bits + 9)
    n = 1001
    for bb in (Broadcast(4, 0), Broadcast(1, 7), Broadcast(3, 5), Broadcast(n, 0)):
        m = broadcast_elements(n, bb)
        a = nb.random_numbers(rng, n, bits, 9)
        b = nb.random_numbers(rng, m, bits, 9)
        out, _ = engine.run(bits, Operation.mul, a, b, b_index=bb)
        assert same(out, oracle.elementwise(bits, 2, a, b, b_index=(bb.stride, bb.period)))
        A, B, O = engine.make_buffer(n, bits), engine.make_buffer(m, bits), engine.make_buffer(n, bits)
        A.upload(a)
        B.upload(b)
        batch = engine.batch()
        batch.run(Operation.div, A, B, None, O, b_index=bb)
        batch.submit().wait()
        assert same(O.download(), oracle.elementwise(bits, 3, a, b, b_index=(bb.stride, bb.period)))
        cb = Broadcast(2, 3)
        mc = broadcast_elements(n, cb)
        x, y, z = nb.random_complex(rng, n, bits, 5), nb.random_complex(rng, m, bits, 5), nb.random_complex(rng, mc, bits, 8)
        out, _ = engine.run(bits, Operation.complex_mul, x, y, b_index=bb)
        assert same(out, oracle.elementwise(bits, 5, x, y, b_index=(bb.stride, bb.period)))
        out, _ = engine.run_ternary(bits, Operation.complex_fma, x, y, z, b_index=bb, c_index=cb)
        assert same(out, oracle.elementwise(bits, 11, x, y, z, b_index=(bb.stride, bb.period), c_index=(cb.stride, cb.period)))


def test_resident_mul_chain_is_fused_and_exact(engine, oracle):
    """Config-1 shape at reduced count: x <- x * f_s, 16 steps at 1024 bits, in one batch; the
    batch fuses the steps into one register-resident kernel."""
    from limbforge_b200.api import Operation
    bits, count, steps = 1024, 4096, 16
    rng = np.random.default_rng(7)
    x = nb.random_numbers(rng, count, bits, 8, zero_frac=0.01, sparse_frac=0.02)
    f = np.stack([nb.random_numbers(rng, count, bits, 8, zero_frac=0.01, sparse_frac=0.02) for _ in range(steps)])
    want = oracle.mul_chain(bits, x, f)
    X = engine.make_buffer(count, bits)
    X.upload(x)
    F = [engine.make_buffer(count, bits) for _ in range(steps)]
    for s in range(steps):
        F[s].upload(f[s])
    batch = engine.batch()
    for s in range(steps):
        batch.run(Operation.mul, X, F[s], None, X)
    t = batch.submit().wait()
    assert same(X.download(), want)
    assert t.gpu_seconds > 0
    # observable intermediates: y1 = x*f0, y2 = y1*f1 written to separate buffers
    Y1, Y2 = engine.make_buffer(count, bits), engine.make_buffer(count, bits)
    X.upload(x)
    batch = engine.batch()
    batch.run(Operation.mul, X, F[0], None, Y1)
    batch.run(Operation.add, Y1, F[1], None, Y2)
    batch.run(Operation.div, Y2, F[2], None, Y2)
    batch.submit().wait()
    y1 = oracle.elementwise(bits, 2, x, f[0])
    y2 = oracle.elementwise(bits, 3, oracle.elementwise(bits, 0, y1, f[1]), f[2])
    assert same(Y1.download(), y1)
    assert same(Y2.download(), y2)


def test_device_pointer_chain_entry(oracle):
    import ctypes
    from limbforge_b200 import api
    bits, count, steps = 512, 3000, 5
    rng = np.random.default_rng(11)
    x = nb.random_numbers(rng, count, bits, 8)
    f = np.stack([nb.random_numbers(rng, count, bits, 8) for _ in range(steps)])
    want = oracle.mul_chain(bits, x, f)
    e = api.Engine()
    X, F, O = e.make_buffer(count, bits), e.make_buffer(count * steps, bits), e.make_buffer(count, bits)
    X.upload(x)
    F.upload(f.reshape(count * steps, -1))
    api.dev_mul_chain(bits, X.device_pointer(), F.device_pointer(), count, steps, O.device_pointer(), count)
    cudart = ctypes.CDLL("libcudart.so")
    assert cudart.cudaDeviceSynchronize() == 0
    assert same(O.download(), want)


def test_buffer_ownership_and_batch_errors(engine):
    """tests/test_buffers.cpp: busy buffers, foreign engines, single-use batches, short operands."""
    from limbforge_b200 import api
    from limbforge_b200.api import Broadcast, InvalidArgument, LogicError, Operation
    bits, n = 256, 64
    rng = np.random.default_rng(2)
    a = nb.random_numbers(rng, n, bits, 9)
    A, B, O = engine.make_buffer(n, bits), engine.make_buffer(n, bits), engine.make_buffer(n, bits)
    A.upload(a)
    B.upload(a)
    batch = engine.batch()
    batch.run(Operation.mul, A, B, None, O)
    sub = batch.submit()
    with pytest.raises(LogicError):
        batch.submit()
    with pytest.raises(LogicError):
        batch.run(Operation.mul, A, B, None, O)
    sub.wait()
    assert sub.ready()
    sub.wait()                                        # repeated waits are fine
    other = api.Engine()
    foreign = other.make_buffer(n, bits)
    with pytest.raises(InvalidArgument):
        b2 = engine.batch()
        b2.run(Operation.add, A, foreign, None, O)
    with pytest.raises(InvalidArgument):
        short = engine.make_buffer(1, bits)
        b3 = engine.batch()
        b3.run(Operation.add, engine.make_buffer(8, bits), short, None, engine.make_buffer(8, bits), b_index=Broadcast(4, 0))
    with pytest.raises(InvalidArgument):
        engine.run(100, Operation.add, a, a)
    with pytest.raises(InvalidArgument):
        engine.run(bits, Operation.fma, a, a)
    with pytest.raises(InvalidArgument):
        engine.run_ternary(bits, Operation.add, a, a, a)
    # mapped(): a host view; writes reach the device at the next submission
    view = A.mapped()
    view[:] = 0
    view[:, bits // 32 - 1] = 0x80000000
    view[:, bits // 32 + 1] = 1                       # every value = 1
    batch = engine.batch()
    batch.run(Operation.mul, A, B, None, O)
    sub = batch.submit()
    with pytest.raises(LogicError):
        A.mapped()
    with pytest.raises(LogicError):
        A.upload(a)
    sub.wait()
    assert same(O.download(), a)
    # empty batches and zero counts are accepted
    engine.batch().submit().wait()
    out, t = engine.run(bits, Operation.add, a[:0], a[:0])
    assert out.shape[0] == 0


def test_dense_1024_complex_repeats(engine, oracle):
    """tests/test_arithmetic.cpp:115-129: 65,536 dense 1024-bit complex values, three GPU repeats."""
    from limbforge_b200.api import Operation
    bits, count = 1024, 65536
    rng = np.random.default_rng(20261007 + bits)
    a = nb.random_complex(rng, count, bits, 5)
    b = nb.random_complex(rng, count, bits, 5)
    for op in (4, 5, 6):
        want = oracle.elementwise(bits, op, a, b)
        for _ in range(3):
            out, _ = engine.run(bits, Operation(op), a, b)
            assert same(out, want), f"op {op} bad {first_bad(out, want)}"
