"""CPU, two gloo ranks: the multi-rank bookkeeping of the batched path.

Each rank partitions a ragged batch of 400 mixed-precision instances and a 1,000,003-value chain.
The test checks that the shares are disjoint and cover everything, that both ranks compute the same
partition, that the ragged loads balance, and that the max over ranks of a per-rank time reaches
every rank."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from limbforge_b200 import api, shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _items():
    rng = np.random.default_rng(9)
    count = 400
    return api.ragged_items(rng.choice([128, 256, 512, 1024], size=count), rng.integers(4, 49, size=count),
                            rng.integers(4, 49, size=count), rng.integers(4, 49, size=count))


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        parts = shard.ragged_partition(_items(), world)
        lo, hi = shard.split_range(1_000_003, rank, world)
        t = shard.max_over_ranks(1.0 + rank * 2.5, dist)
        # every rank sends its view to rank 0
        mine = torch.tensor(np.concatenate([parts[rank], [-1, lo, hi]]), dtype=torch.int64)
        sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(sizes, torch.tensor([mine.numel()]))
        buf = [torch.zeros(int(s.item()), dtype=torch.int64) for s in sizes]
        dist.all_gather(buf, mine)
        out.put((rank, t, [b.numpy().tolist() for b in buf]))
    finally:
        dist.destroy_process_group()


def _gemm_rank(rank, world, port, out):
    from oracle.oracle import Oracle
    from limbforge_b200 import numbers as nb
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        orc = Oracle()
        rng = np.random.default_rng(21)
        bits, m, n, k = 128, 37, 9, 11
        A = nb.random_numbers(rng, k * m, bits, 40)
        B = nb.random_numbers(rng, k * n, bits, 40)
        C = nb.random_numbers(rng, m * n, bits, 40)

        def gemm(bits_, ta, a, b, rows, n_, k_, c, sub):      # the per-rank product (Linalg.gemm on a GPU)
            c[:] = orc.gemm(bits_, ta, a, b, rows, n_, k_, c, sub)
        got = shard.sharded_exact_gemm(gemm, bits, True, A, B, m, n, k, C, True, dist, align=8)
        got2 = shard.sharded_exact_gemm(gemm, bits, False, A, B, m, n, k, None, False, dist, align=8)
        out.put((rank, got, got2))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_sharded_exact_gemm():
    """Row blocks of an exact product on two ranks, all-gathered, equal the whole product bit for bit."""
    from oracle.oracle import Oracle
    from limbforge_b200 import numbers as nb
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gemm_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    orc = Oracle()
    rng = np.random.default_rng(21)
    bits, m, n, k = 128, 37, 9, 11
    A = nb.random_numbers(rng, k * m, bits, 40)
    B = nb.random_numbers(rng, k * n, bits, 40)
    C = nb.random_numbers(rng, m * n, bits, 40)
    want = orc.gemm(bits, True, A, B, m, n, k, C, True)
    want2 = orc.gemm(bits, False, A, B, m, n, k)
    for _, got, got2 in results:
        assert (got == want).all() and (got2 == want2).all()
    assert shard.gemm_row_block(37, 0, 2, 8) == (0, 24) and shard.gemm_row_block(37, 1, 2, 8) == (24, 37)


def test_two_gloo_ranks_partition_and_max():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    items = _items()
    for rank, t, views in results:
        assert t == pytest.approx(3.5)                      # max over ranks of 1.0 and 3.5
        idx = [np.array(v[:-3]) for v in views]
        ranges = [tuple(v[-2:]) for v in views]
        allidx = np.sort(np.concatenate(idx))
        assert (allidx == np.arange(len(items))).all()      # disjoint and complete
        assert ranges[0][0] == 0 and ranges[-1][1] == 1_000_003 and ranges[0][1] == ranges[1][0]
        cost = shard.ragged_cost(items)
        loads = [cost[i].sum() for i in idx]
        assert max(loads) <= cost.sum() / world + cost.max() + 1e-6
    assert results[0][2] == results[1][2]                   # both ranks saw the same partition


def test_split_range_and_partition_single_process():
    assert shard.split_range(10, 0, 3) == (0, 4) and shard.split_range(10, 2, 3) == (7, 10)
    assert shard.split_range(0, 1, 4) == (0, 0)
    with pytest.raises(ValueError):
        shard.split_range(5, 3, 3)
    parts = shard.ragged_partition(_items(), 1)
    assert len(parts) == 1 and len(parts[0]) == 400
    assert shard.max_over_ranks(2.0) == 2.0
