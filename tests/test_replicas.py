"""Replica parallelism on CPU: sharding balance and the max-over-ranks timing reduction with
two gloo ranks (the GPU bench uses the same helpers over NCCL)."""
import os
import socket

import numpy as np
import pytest

from galsim_b200 import replicas


def test_shard_partitions_and_balances():
    rng = np.random.default_rng(3)
    N = rng.choice([128, 192, 256, 384, 512], size=4097, p=[0.8, 0.15, 0.03, 0.015, 0.005])
    for world in (1, 2, 3, 8):
        parts = [replicas.shard(N, r, world) for r in range(world)]
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(len(N)))
        cost = [replicas.stamp_cost(N[p]).sum() for p in parts]
        assert max(cost) - min(cost) <= replicas.stamp_cost(512)
        for size in np.unique(N):
            counts = [np.sum(N[p] == size) for p in parts]
            assert max(counts) - min(counts) <= 1


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    r, w = replicas.init('gloo', timeout_s=30)
    assert (r, w) == (rank, world)
    replicas.barrier()
    local_ms = 10. + 5. * rank
    out.put((rank, replicas.max_over_ranks(local_ms), len(replicas.shard(np.full(10, 128), rank, world))))
    replicas.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=60) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]
    assert [r[2] for r in res] == [5, 5]
