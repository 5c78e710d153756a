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


def _logdet_of(i, orders, seeds):
    from oracle import restated

    n = int(orders[i])
    g = np.random.default_rng(int(seeds[i]))
    G = g.standard_normal((n, n))
    F, info = restated.potrf(G @ G.T / n + 0.1 * np.eye(n), "L")
    return (2.0 * restated.diag_logdet(np.tril(F)).real if info == 0 else float("nan")), info


def _worker(rank, world, port, orders, seeds, out):
    import torch
    import torch.distributed as dist

    from libddla_b200.ddla.batched import sharded_run

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seen = []

        def compute(idx):
            seen.extend(idx)
            return torch.tensor([_logdet_of(i, orders, seeds) for i in idx], dtype=torch.float64).reshape(-1, 2)

        merged = sharded_run(orders, compute)
        out.put((rank, sorted(seen), merged.numpy()))
    finally:
        dist.destroy_process_group()


def test_sharded_batch_over_two_gloo_ranks():
    """sharded_run on two gloo ranks: each rank computes only its LPT shard, and
    both end with every matrix's (logdet, info) in batch order, equal to the
    single-process answer."""
    import socket

    import torch.multiprocessing as mp

    rng = np.random.default_rng(9)
    orders = rng.integers(2, 40, size=25)
    seeds = rng.integers(0, 2**31, size=25)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, orders, seeds, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards = shard_lpt(orders, 2)
    want = np.array([_logdet_of(i, orders, seeds) for i in range(len(orders))])
    for rank, seen, merged in results:
        assert seen == sorted(shards[rank])  # each rank computed only its shard
        assert merged.shape == (len(orders), 2)
        np.testing.assert_array_equal(merged[:, 1], want[:, 1])
        np.testing.assert_allclose(merged[:, 0], want[:, 0], rtol=1e-12, atol=0)


def test_sharded_run_single_process():
    import torch

    from libddla_b200.ddla.batched import sharded_run

    orders = np.array([5, 1, 9, 3])
    out = sharded_run(orders, lambda idx: torch.tensor([float(orders[i]) ** 2 for i in idx]))
    assert out.shape == (4, 1)
    assert out[:, 0].tolist() == [25.0, 1.0, 81.0, 9.0]
    with pytest.raises(ValueError):
        sharded_run(orders, lambda idx: torch.zeros(len(idx) + 1, 1))
