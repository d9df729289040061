"""Sharding of independent instances over ranks: the cost-balanced split and
the gather back into global order, on world_size 2 with the gloo backend on
CPU (the same calls run over NCCL on GPUs)."""
import os
import socket

import numpy as np
import pytest
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
