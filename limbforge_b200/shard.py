"""Sharding of the batched path over ranks (one process per GPU).

Every workload of this path is a set of independent units: values of an element-wise op or a chain,
instances of a ragged GEMM batch, systems of a batched 4x4 LU, or rows of an exact product's output.
Ranks therefore take disjoint units and exchange nothing while they compute. The only
collectives are bookkeeping: the max over ranks of the device time, and gathering results where
a caller wants them on one rank."""
from __future__ import annotations

import numpy as np


def split_range(count: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous share [lo, hi) of `count` units for `rank`; sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(count, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def ragged_cost(items: np.ndarray) -> np.ndarray:
    """Work of each ragged GEMM instance: m n k products of (bits/32)^2 word products each."""
    limbs = items["bits"].astype(np.float64) / 32.0
    return items["m"].astype(np.float64) * items["n"] * items["k"] * limbs * limbs


def ragged_partition(items: np.ndarray, world: int) -> list[np.ndarray]:
    """Instance indices per rank, balanced by cost. The greedy assignment takes the instances in
    decreasing cost and gives each to the least loaded rank; the heaviest rank then carries at most
    the mean load plus one instance's cost. Ties are broken by index, so every rank computes the same
    partition."""
    if world < 1:
        raise ValueError("world must be positive")
    cost = ragged_cost(items)
    order = np.lexsort((np.arange(cost.size), -cost))
    load = np.zeros(world)
    owner = np.empty(cost.size, dtype=np.int64)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += cost[i]
    return [np.nonzero(owner == r)[0] for r in range(world)]


def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """The maximum of `value` over all ranks of the default process group (the value itself when
    there is no group): the job's time is its slowest rank's."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gemm_row_block(m: int, rank: int, world: int, align: int = 128) -> tuple[int, int]:
    """Rows [lo, hi) of an m-row exact product's output for `rank`: whole blocks of `align` rows (the residue engine's
    output tile height) split as evenly as split_range splits units, the last block ragged."""
    if align < 1:
        raise ValueError("align must be positive")
    blocks = (m + align - 1) // align
    lo, hi = split_range(blocks, rank, world)
    return min(m, lo * align), min(m, hi * align)


def sharded_exact_gemm(gemm, bits: int, transpose_a: bool, A: np.ndarray, B: np.ndarray, m: int, n: int, k: int,
                       C: np.ndarray | None = None, subtract: bool = False, dist=None, align: int = 128) -> np.ndarray:
    """C <- RN(C - op(A) B) (or RN(op(A) B)) with C's rows split over the ranks of the default process group: each rank
    computes its row block with `gemm(bits, transpose_a, A_rows, B, rows, n, k, C_rows, subtract)` (Linalg.gemm, or any
    function of that signature) from op(A)'s matching rows and all of B, and an all-gather assembles the whole C on
    every rank.  Every output is one rounding of its own exact dot product, so the result is bit-identical to the
    unsharded product whatever the split.  Arrays are element words: A [k*m or m*k, W], B [k*n, W], C [m*n, W]."""
    w = A.shape[-1]
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    lo, hi = gemm_row_block(m, rank, world, align)
    rows = hi - lo
    if transpose_a:
        a_rows = np.ascontiguousarray(A.reshape(k, m, w)[:, lo:hi]).reshape(k * rows, w)
    else:
        a_rows = np.ascontiguousarray(A.reshape(m, k, w)[lo:hi]).reshape(rows * k, w)
    c_rows = (np.zeros((rows * n, w), np.uint32) if C is None else
              np.ascontiguousarray(C.reshape(m, n, w)[lo:hi]).reshape(rows * n, w))
    if rows:
        gemm(bits, transpose_a, a_rows, B, rows, n, k, c_rows, subtract)
    if world == 1:
        return c_rows
    import torch
    most = max(gemm_row_block(m, r, world, align)[1] - gemm_row_block(m, r, world, align)[0] for r in range(world))
    mine = torch.zeros((most * n, w), dtype=torch.int32)
    mine[:rows * n] = torch.from_numpy(c_rows.view(np.int32))
    parts = [torch.zeros_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine)
    out = np.empty((m * n, w), np.uint32)
    for r, t in enumerate(parts):
        a, b = gemm_row_block(m, r, world, align)
        out[a * n:b * n] = t[:(b - a) * n].numpy().view(np.uint32)
    return out
