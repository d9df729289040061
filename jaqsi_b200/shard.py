"""Sharding of independent instances over ranks (one process per GPU).

The batched workloads (many parameter sets, or many uneven circuits) are
independent per instance, so ranks split the instances with no data-path
exchange: each rank runs its share through its own GPU, then the per-instance
results are gathered back into the global order.  This mirrors the
reference's batch ``shard_map`` over devices (jaqsi/script.py:87-125),
which splits the batch axis evenly; here the split balances the estimated
cost (2^n x blocks per instance), since uneven circuits differ by orders of
magnitude.

Only the gather of results touches the process group (``all_gather_object``,
any backend: NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import heapq
from typing import Callable, List, Optional, Sequence, Tuple

__all__ = ["partition", "instance_cost", "run_sharded"]


def instance_cost(n_qubits: int, n_ops: int) -> float:
    """Relative cost of one forward + adjoint instance: every op is a pass over
    2^n amplitudes."""
    return float(1 << int(n_qubits)) * max(1, int(n_ops))


def partition(costs: Sequence[float], world: int) -> List[List[int]]:
    """Greedy longest-processing-time split of instance indices over `world`
    ranks: instances in descending cost order, each to the currently least
    loaded rank (ties to the lowest rank).  Deterministic, so every rank
    computes the same split without communicating.  Each rank's indices are
    returned in ascending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    shares: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shares]


def run_sharded(costs: Sequence[float], local_fn: Callable[[List[int]], list], group=None,
                rank: Optional[int] = None, world: Optional[int] = None) -> list:
    """Run `local_fn` on this rank's share of the instances and return the
    per-instance results of all ranks in global instance order.

    ``local_fn(indices)`` returns one result per index, in the order given.
    Without an initialised process group (or with world 1) it runs locally.
    """
    import torch.distributed as dist

    if world is None:
        world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    if rank is None:
        rank = dist.get_rank(group) if world > 1 else 0
    shares = partition(costs, world)
    mine = shares[rank]
    local = list(local_fn(mine))
    if len(local) != len(mine):
        raise ValueError(f"local_fn returned {len(local)} results for {len(mine)} instances")
    if world == 1:
        return local
    gathered: List[Tuple[List[int], list]] = [None] * world  # type: ignore[list-item]
    dist.all_gather_object(gathered, (mine, local), group=group)
    out: list = [None] * len(costs)
    for idx, res in gathered:
        for i, r in zip(idx, res):
            out[i] = r
    return out
