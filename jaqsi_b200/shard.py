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

Batched ``Script.execute(..., in_axes=...)`` calls shard the same way inside
``batch_sharding()``: every rank passes the same logical batch, runs a
contiguous slice of it (the reference's ``shard_map`` splits the batch axis
evenly, jaqsi/script.py:87-125), and the slices are all-gathered into the
full result on every rank (one tensor collective).  In the backward pass the
gradient of the full result is identical on every rank; each rank pulls its
own rows back through its kernels, and one all-reduce (sum) per argument
tensor adds the ranks' contributions, so every rank holds the full gradient
of broadcast (``in_axes=None``) and batched arguments alike, as the reference's
transpose sums the replicated cotangent (:114-119).
"""
from __future__ import annotations

import contextlib
import heapq
import threading
from typing import Callable, List, Optional, Sequence, Tuple

import torch

__all__ = ["partition", "instance_cost", "run_sharded", "batch_sharding", "active", "row_range",
           "sharded_batch_call"]


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


# ---------------------------------------------------------------------------
# batched Script calls split over ranks
# ---------------------------------------------------------------------------
_STATE = threading.local()


@contextlib.contextmanager
def batch_sharding(group=None):
    """Within the block, batched ``Script.execute`` calls (``in_axes``) on this
    thread split their batch over the ranks of ``group`` (default: the world
    group).  Every rank must make the same calls with the same batch."""
    prev = getattr(_STATE, "group", None), getattr(_STATE, "on", False)
    _STATE.group, _STATE.on = group, True
    try:
        yield
    finally:
        _STATE.group, _STATE.on = prev


@contextlib.contextmanager
def _suspended():
    """Batch sharding off inside (the per-rank share runs unsharded)."""
    prev = getattr(_STATE, "on", False)
    _STATE.on = False
    try:
        yield
    finally:
        _STATE.on = prev


def active():
    """(group, rank, world) when batch sharding is on and the group has more
    than one rank, else None."""
    if not getattr(_STATE, "on", False):
        return None
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return None
    group = _STATE.group
    world = dist.get_world_size(group)
    if world < 2:
        return None
    return group, dist.get_rank(group), world


def row_range(batch: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous rows [lo, hi) of rank `rank`: the first batch % world ranks
    take one row more."""
    base, extra = divmod(batch, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


class _SumGrad(torch.autograd.Function):
    """Identity forward; backward all-reduces (sums) the gradient over the group."""

    @staticmethod
    def forward(ctx, x, group):
        ctx.group = group
        return x.view_as(x)

    @staticmethod
    def backward(ctx, g):
        import torch.distributed as dist

        g = g.contiguous().clone()
        dist.all_reduce(_real(g), op=dist.ReduceOp.SUM, group=ctx.group)
        return g, None


class _GatherRows(torch.autograd.Function):
    """All-gather of each rank's rows (padded to the largest share) into the
    full batch; backward returns this rank's rows of the incoming gradient."""

    @staticmethod
    def forward(ctx, y, group, rank, world, batch):
        import torch.distributed as dist

        ctx.rows = row_range(batch, rank, world)
        size = row_range(batch, 0, world)[1]  # the largest share (rank 0's)
        pad = torch.zeros((size,) + tuple(y.shape[1:]), dtype=y.dtype, device=y.device)
        pad[: y.shape[0]] = y
        out = torch.empty((world * size,) + tuple(y.shape[1:]), dtype=y.dtype, device=y.device)
        dist.all_gather_into_tensor(_real(out), _real(pad), group=group)
        full = torch.cat([out[r * size: r * size + (row_range(batch, r, world)[1] - row_range(batch, r, world)[0])]
                          for r in range(world)])
        return full

    @staticmethod
    def backward(ctx, g):
        lo, hi = ctx.rows
        return g[lo:hi], None, None, None, None


def _real(t: torch.Tensor) -> torch.Tensor:
    return torch.view_as_real(t) if t.is_complex() else t


def sharded_batch_call(local_fn: Callable, args: tuple, in_axes: tuple, batch: int, group, rank: int, world: int,
                       initial_state=None):
    """Run ``local_fn(local_args, local_batch, local_initial_state)`` on this
    rank's rows and return the full-batch result on every rank.

    Tensor arguments that need gradients pass through an all-reduce of their
    gradient first; batched arguments (and a 2-D initial state) are then cut
    to this rank's rows along their batch axis, broadcast ones are passed
    whole."""
    lo, hi = row_range(batch, rank, world)
    local = []
    for a, ax in zip(args, in_axes):
        if isinstance(a, torch.Tensor) and a.requires_grad:
            a = _SumGrad.apply(a, group)
        if isinstance(a, torch.Tensor) and ax is not None:
            a = a.narrow(ax, lo, hi - lo)
        local.append(a)
    init = initial_state
    if isinstance(init, torch.Tensor):
        if init.requires_grad:
            init = _SumGrad.apply(init, group)
        if init.dim() == 2:
            init = init[lo:hi]
    with _suspended():
        y = local_fn(tuple(local), hi - lo, init)
    return _GatherRows.apply(y, group, rank, world, batch)
