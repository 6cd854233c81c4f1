"""Multi-GPU sweep: independent (ROM, frequency) systems, sharded across ranks.

Every system of the sweep is independent, so ranks need no collective on the data path:
each rank owns a set of ROMs (or frequency ranges), sweeps them on its own GPU and the host
gathers results only if it wants them.  The only collectives are the barrier and the
max-over-ranks of the step time used by the benchmark.

* ``partition(costs, world)``      longest-processing-time greedy split of work items by cost
                                    (cost of a ROM = F * (8/3 n^3 + 8 n^2 r)), one list per rank;
* ``rom_cost(n, r, F)``            the algorithmic flop count used as the cost;
* ``rank_seed(base, rank)``        per-rank workload seed for weak scaling (each GPU sweeps its
                                    own batch of ROMs of the same distribution);
* ``max_over_ranks(x, group)``     the step-time reduction (works on gloo and nccl);
* ``frequency_slice(F, world, rank)``  the contiguous block of frequencies a rank takes in a
                                    sharded full-order sweep (``krylov.fom_sweep``: every frequency
                                    is its own factorisation, so frequencies shard with no
                                    collective; sizes differ by at most one).

The Krylov basis process does not shard: each expansion point's blocks are re-orthogonalised
against every column before them.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def rom_cost(n: int, r: int, F: int) -> float:
    return F * (8.0 / 3.0 * n ** 3 + 8.0 * n * n * r)


def partition(costs: Sequence[float], world: int) -> List[List[int]]:
    """Greedy LPT partition: items sorted by decreasing cost go to the least-loaded rank.
    Deterministic (ties broken by rank index, then item index)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, k) for k in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, k = heapq.heappop(heap)
        out[k].append(i)
        heapq.heappush(heap, (load + costs[i], k))
    return [sorted(x) for x in out]


def rank_seed(base: int, rank: int) -> int:
    return base + 1000003 * rank


def max_over_ranks(x: float, group=None, device=None) -> float:
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def frequency_slice(n_freq: int, world: int, rank: int):
    """(start, stop) of rank's contiguous share of n_freq frequencies: the first n_freq % world
    ranks take one more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    q, rem = divmod(n_freq, world)
    start = rank * q + min(rank, rem)
    return start, start + q + (1 if rank < rem else 0)
