"""Sharding of batched work over ranks (one process per GPU): the LPT partition
covers every matrix exactly once with balanced cost, and world-size-2 gloo
ranks that each process their shard and gather the per-matrix results reproduce
the single-process answer (CPU only: the per-matrix work here is the oracle)."""
import os

import numpy as np
import pytest

from libddla_b200.ddla.batched import shard_lpt


def test_shard_lpt_partition_and_balance():
    rng = np.random.default_rng(4)
    orders = rng.integers(16, 513, size=4096)
    for world in (1, 2, 3, 8):
        shards = shard_lpt(orders, world)
        allidx = sorted(i for s in shards for i in s)
        assert allidx == list(range(len(orders)))
        loads = [sum(float(orders[i]) ** 3 for i in s) for s in shards]
        assert max(loads) - min(loads) <= float(orders.max()) ** 3
    with pytest.raises(ValueError):
        shard_lpt(orders, 0)


def _worker(rank, world, port, orders, seeds, out):
    import torch
    import torch.distributed as dist

    from oracle import restated

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard_lpt(orders, world)[rank]
        res = torch.full((len(orders),), float("nan"), dtype=torch.float64)
        for i in mine:
            n = int(orders[i])
            g = np.random.default_rng(int(seeds[i]))
            G = g.standard_normal((n, n))
            F, info = restated.potrf(G @ G.T / n + 0.1 * np.eye(n), "L")
            res[i] = 2.0 * restated.diag_logdet(np.tril(F)).real if info == 0 else float("nan")
        gathered = [torch.empty_like(res) for _ in range(world)]
        dist.all_gather(gathered, res)
        merged = torch.stack(gathered).nan_to_num(nan=0.0).sum(0)
        if rank == 0:
            out.put(merged.numpy())
    finally:
        dist.destroy_process_group()


def test_sharded_batch_over_two_gloo_ranks():
    import socket

    import torch.multiprocessing as mp

    rng = np.random.default_rng(9)
    orders = rng.integers(2, 40, size=24)
    seeds = rng.integers(0, 2**31, size=24)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, orders, seeds, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from oracle import restated

    for i, n in enumerate(orders):
        g = np.random.default_rng(int(seeds[i]))
        G = g.standard_normal((n, n))
        F, info = restated.potrf(G @ G.T / n + 0.1 * np.eye(n), "L")
        assert info == 0
        assert abs(merged[i] - 2.0 * restated.diag_logdet(np.tril(F)).real) < 1e-12 * max(1.0, abs(merged[i]))
