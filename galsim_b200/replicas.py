"""Replica parallelism for the FFT drawing path: one process per GPU, stamps sharded across
ranks with no collective on the data path (stamps are independent; the reference draws them
one by one in separate processes, galsim/config/util.py:672).

* shard(N, rank, world) -- a size-balanced partition of a batch by stamp: stamps are dealt
  round-robin in order of decreasing cost (N^2 log2 N of their FFT size), so every rank gets a
  similar share of the work when the sizes are uneven.
* max_over_ranks(x) -- the reduction used for timing (the slowest rank sets the job time).
* launch environment: RANK / WORLD_SIZE / LOCAL_RANK from torchrun, 127.0.0.1 rendezvous.
"""
import os

import numpy as np


def rank_info():
    """(rank, world, local_rank) from the torchrun environment (1 process: 0, 1, 0)."""
    return (int(os.environ.get('RANK', '0')), int(os.environ.get('WORLD_SIZE', '1')),
            int(os.environ.get('LOCAL_RANK', '0')))


def init(backend='nccl', timeout_s=120):
    """Initialise the process group when running under torchrun (world > 1)."""
    import datetime
    import torch.distributed as dist
    rank, world, _ = rank_info()
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world


def stamp_cost(N):
    N = np.asarray(N, np.float64)
    return N * N * np.log2(np.maximum(N, 2.))


def shard(N, rank, world):
    """Indices of the stamps that `rank` draws: round-robin over the stamps sorted by
    decreasing FFT cost (ties by index), so per-rank work differs by at most one stamp of each
    size class."""
    N = np.asarray(N)
    order = np.lexsort((np.arange(len(N)), -stamp_cost(N)))
    return np.sort(order[rank::world])


def max_over_ranks(x):
    """The maximum of a float over all ranks (x itself with one process)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64)
    if dist.get_backend() == 'nccl':
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
