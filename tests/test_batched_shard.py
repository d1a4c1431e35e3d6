"""Sharding of the batched uneven solves over several GPUs (host side, CPU):
the cost partition and the final gather run as world_size-2 gloo ranks.
The systems are independent, so these are the only cross-rank steps."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from charmlu_b200.batched import gather_results, log_uniform_orders, partition_by_cost


def test_partition_covers_and_balances():
    n = log_uniform_orders(4096, 32, 1024, seed=42)
    cost = (2.0 / 3.0) * n.astype(np.float64) ** 3 + 2.0 * n.astype(np.float64) ** 2
    for parts in (1, 2, 3, 8):
        p = partition_by_cost(n, parts)
        allidx = np.concatenate(p)
        assert sorted(allidx.tolist()) == list(range(len(n)))
        loads = np.array([cost[q].sum() for q in p])
        # LPT: the heaviest part exceeds the mean by at most one system's cost
        assert loads.max() - loads.mean() <= cost.max() + 1e-6
        assert loads.max() / loads.mean() < 1.01
    assert all(np.array_equal(a, b) for a, b in zip(partition_by_cost(n, 4), partition_by_cost(n, 4)))


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = log_uniform_orders(300, 32, 1024, seed=7)
        mine = partition_by_cost(n, world)[rank]
        info = (mine % 3 == 0).astype(np.int64) * (mine + 1)   # a fake singular status on every third system
        res = n[mine] * 1e-3
        g_info, g_res = gather_results(mine, info, res, len(n))
        idx = np.arange(len(n))
        ok = (np.array_equal(g_info, (idx % 3 == 0) * (idx + 1)) and np.allclose(g_res, n * 1e-3))
        q.put((rank, bool(ok)))
    finally:
        dist.destroy_process_group()


def test_gather_results_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert out == {0: True, 1: True}
