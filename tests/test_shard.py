"""Multi-rank host logic on CPU: world-size-2 gloo process groups.

The GPU paths shard batches by system and run single systems as replicas;
what crosses ranks is host-side (the partition, the max-over-ranks timing and
the report gather), so it is exercised here without a GPU.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cholesky_gpu_b200 import matgen
from cholesky_gpu_b200.shard import gather_by_system, max_over_ranks, partition_systems, shard_cost


def test_partition_covers_every_system_once_and_balances():
    ns = [int(v) for v in matgen.batch_sizes(512, 64, 2048, 8)]
    for world in (1, 2, 4, 8):
        shards = partition_systems(ns, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(ns)))
        costs = [shard_cost(ns, s) for s in shards]
        # LPT bound: max load <= mean load + largest single job
        assert max(costs) <= np.mean(costs) + max(n ** 3 for n in ns)
        assert partition_systems(ns, world) == shards          # deterministic


def test_partition_edge_cases():
    assert partition_systems([100], 4) == [[0], [], [], []]
    assert partition_systems([], 2) == [[], []]
    with pytest.raises(ValueError):
        partition_systems([1], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, ns, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shard = partition_systems(ns, world)[rank]
        # each rank "solves" its systems: a result that names the system and the rank
        local = {i: (i, rank, ns[i]) for i in shard}
        allres = gather_by_system(local, len(ns), dist)
        t = max_over_ranks(float(10 * (rank + 1)), dist)
        q.put((rank, allres, t))
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_and_max_over_ranks_with_gloo():
    ns = [int(v) for v in matgen.batch_sizes(37, 64, 2048, 3)]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, ns, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards = partition_systems(ns, world)
    for rank, allres, t in out:
        assert t == 20.0                                     # max over the two ranks
        assert [r[0] for r in allres] == list(range(len(ns)))
        for i, owner, n in allres:
            assert i in shards[owner] and n == ns[i]
