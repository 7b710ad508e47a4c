"""Multi-GPU path of the batching form, on the CPU: two gloo ranks each take
their cost-balanced shard of the benchmark batch (no data exchange); the
shards partition the batch and balance its FLOPs, and the timing reduction is
the max over ranks.  The plain and precision forms run as independent
replicas (no collective on the data path), which needs no test beyond the
single-GPU ones."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

import lu2_b200 as L


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import lu2_b200 as L2

        n, r = L2.batch_sizes(20000, 1, 16, 512, 0.1, 8)
        idx = L2.batch_shard(n, r, world, rank)
        parts = [None] * world
        dist.all_gather_object(parts, idx.tolist())
        t = torch.tensor([0.5 + rank], dtype=torch.float64)  # this rank's "device time"
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
        if rank == 0:
            q.put((parts, float(t.item())))
    finally:
        dist.destroy_process_group()


def test_batch_shard_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        parts, tmax = q.get(timeout=180)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    a, b = set(parts[0]), set(parts[1])
    assert not (a & b) and sorted(a | b) == list(range(20000))
    n, r = L.batch_sizes(20000, 1, 16, 512, 0.1, 8)
    cost = 2.0 / 3.0 * n.astype(float) ** 3 + 2.0 * n.astype(float) ** 2 * r
    ca, cb = cost[sorted(a)].sum(), cost[sorted(b)].sum()
    assert abs(ca - cb) / max(ca, cb) < 1e-3
    assert tmax == 1.5


@pytest.mark.parametrize("world", [1, 3, 8])
def test_batch_shard_partitions(world):
    n, r = L.batch_sizes(5000, 2, 16, 512, 0.1, 8)
    shards = [L.batch_shard(n, r, world, k) for k in range(world)]
    allidx = np.concatenate(shards)
    assert np.array_equal(np.sort(allidx), np.arange(5000))
    cost = 2.0 / 3.0 * n.astype(float) ** 3 + 2.0 * n.astype(float) ** 2 * r
    loads = [cost[s].sum() for s in shards]
    assert (max(loads) - min(loads)) / max(loads) < 0.01


def test_batch_shard_rejects_bad_rank():
    with pytest.raises(ValueError):
        L.batch_shard([16, 32], [1, 1], 2, 2)
