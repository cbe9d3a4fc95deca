"""Replica sharding over two CPU ranks (gloo): every instance is inverted
exactly once, results gathered from both ranks match the oracle, and the
timing reduction is a MAX over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from bsofi_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world_size, port, out):
    import torch
    import torch.distributed as dist
    import oracle
    from bsofi_b200.hubbard import random_pcyclic
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    specs = [(3, 4, 1), (5, 3, 2), (2, 6, 3), (4, 4, 4), (6, 2, 5)]
    costs = [n ** 3 * L * L for n, L, _ in specs]
    mine = replicas.shard_by_cost(costs, rank, world_size)
    res = {}
    for i in mine:
        n, L, seed = specs[i]
        M = random_pcyclic(n, L, seed=seed)
        res[i] = oracle.port_inverse(M, n, L)
    gathered = [None] * world_size
    dist.all_gather_object(gathered, res)
    tmax = replicas.max_over_ranks(float(rank + 1))
    replicas.barrier()
    if rank == 0:
        out.put((gathered, tmax))
    dist.destroy_process_group()


def test_shard_partitions():
    for count in (0, 1, 5, 16, 17):
        for w in (1, 2, 3, 8):
            got = sorted(i for r in range(w) for i in replicas.shard(count, r, w))
            assert got == list(range(count))
    costs = [5.0, 1.0, 3.0, 3.0, 2.0]
    parts = [replicas.shard_by_cost(costs, r, 2) for r in range(2)]
    assert sorted(parts[0] + parts[1]) == list(range(5))


@pytest.mark.timeout(180)
def test_two_rank_gloo_replicas():
    from bsofi_b200.hubbard import random_pcyclic
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, tmax = q.get(timeout=150)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert tmax == 2.0
    merged = {}
    for part in gathered:
        assert not (set(part) & set(merged))
        merged.update(part)
    specs = [(3, 4, 1), (5, 3, 2), (2, 6, 3), (4, 4, 4), (6, 2, 5)]
    assert sorted(merged) == list(range(len(specs)))
    for i, (n, L, seed) in enumerate(specs):
        M = random_pcyclic(n, L, seed=seed)
        assert np.linalg.norm(M @ merged[i] - np.eye(n * L)) < 1e-10
