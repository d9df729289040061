"""Sharding of independent instances over ranks: the cost-balanced split and
the gather back into global order, on world_size 2 with the gloo backend on
CPU (the same calls run over NCCL on GPUs)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from jaqsi_b200.shard import instance_cost, partition, run_sharded


def test_partition_covers_everything_once_and_balances():
    rng = np.random.default_rng(4)
    costs = [instance_cost(int(rng.integers(6, 17)), int(rng.integers(10, 41)) * 32) for _ in range(4096)]
    for world in (1, 2, 3, 8):
        shares = partition(costs, world)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shares]
        # LPT bound: max load <= mean + largest single cost
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-6
        assert shares == partition(costs, world)  # deterministic on every rank


def test_partition_edge_cases():
    assert partition([], 2) == [[], []]
    assert partition([5.0], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        partition([1.0], 0)


def test_run_sharded_single_process():
    costs = [3.0, 1.0, 2.0]
    assert run_sharded(costs, lambda idx: [10 * i for i in idx]) == [0, 10, 20]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, costs, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seen = []

        def local(idx):
            seen.extend(idx)
            return [(i, rank, costs[i] * 2) for i in idx]

        out = run_sharded(costs, local)
        q.put((rank, sorted(seen), out))
    finally:
        dist.destroy_process_group()


def test_run_sharded_gloo_world2():
    costs = [float(c) for c in np.random.default_rng(7).integers(1, 1000, 37)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        rank, seen, out = q.get(timeout=120)
        res[rank] = (seen, out)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shares = partition(costs, 2)
    for r in range(2):
        seen, out = res[r]
        assert seen == shares[r]  # each rank computed only its share
        assert [o[0] for o in out] == list(range(len(costs)))  # global order
        assert [o[2] for o in out] == [c * 2 for c in costs]
        assert [o[1] for o in out] == [0 if i in shares[0] else 1 for i in range(len(costs))]


# ---------------------------------------------------------------------------
# batched calls split over ranks: rows, all-gather, gradient all-reduce
# ---------------------------------------------------------------------------
def test_row_ranges_cover_the_batch():
    from jaqsi_b200.shard import row_range

    for batch in (2, 5, 64, 65):
        for world in (2, 3, 8):
            if batch < world:
                continue
            rows = [row_range(batch, r, world) for r in range(world)]
            assert rows[0][0] == 0 and rows[-1][1] == batch
            assert all(rows[r][1] == rows[r + 1][0] for r in range(world - 1))
            assert max(h - l for l, h in rows) - min(h - l for l, h in rows) <= 1


def _stand_in(largs, lbatch, linit):
    """CPU stand-in for one rank's kernel call: a differentiable function of
    batched rows x [b, 3], a broadcast weight w [3] and an initial state."""
    x, w, c = largs
    assert x.shape[0] == lbatch
    base = torch.stack([torch.sin(x @ w) * c, torch.cos(x).sum(-1) * w.sum()], dim=-1)
    if linit is not None:
        base = base + (linit.abs() ** 2).sum(-1, keepdim=True) * w[0]
    return base


def _shard_worker(rank, world, port, batch, q):
    import torch

    from jaqsi_b200 import shard

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = torch.Generator().manual_seed(3)
        x = torch.randn(batch, 3, dtype=torch.float64, generator=g).requires_grad_(True)
        w = torch.randn(3, dtype=torch.float64, generator=g).requires_grad_(True)
        init = torch.randn(batch, 4, dtype=torch.complex128, generator=g).requires_grad_(True)
        ct = torch.randn(batch, 2, dtype=torch.float64, generator=g)
        with shard.batch_sharding():
            spec = shard.active()
            assert spec is not None and spec[1:] == (rank, world)
            y = shard.sharded_batch_call(_stand_in, (x, w, 0.5), (0, None, None), batch, *spec, initial_state=init)
        (y * ct).sum().backward()
        q.put((rank, y.detach().numpy(), x.grad.numpy(), w.grad.numpy(), init.grad.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("batch", [6, 7])
def test_sharded_batch_call_gloo_world2(batch):
    import torch

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, batch, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r = q.get(timeout=120)
        res[r[0]] = r[1:]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # the same computation unsharded in this process
    g = torch.Generator().manual_seed(3)
    x = torch.randn(batch, 3, dtype=torch.float64, generator=g).requires_grad_(True)
    w = torch.randn(3, dtype=torch.float64, generator=g).requires_grad_(True)
    init = torch.randn(batch, 4, dtype=torch.complex128, generator=g).requires_grad_(True)
    ct = torch.randn(batch, 2, dtype=torch.float64, generator=g)
    y = _stand_in((x, w, 0.5), batch, init)
    (y * ct).sum().backward()
    for r in range(2):
        ys, gx, gw, gi = res[r]
        np.testing.assert_allclose(ys, y.detach().numpy(), atol=1e-14)  # full batch on every rank
        np.testing.assert_allclose(gx, x.grad.numpy(), atol=1e-14)
        np.testing.assert_allclose(gw, w.grad.numpy(), atol=1e-14)  # broadcast argument: summed over ranks
        np.testing.assert_allclose(gi, init.grad.numpy(), atol=1e-14)
