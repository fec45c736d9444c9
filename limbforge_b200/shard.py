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
