"""The replica (weak-scaling) path of bench.py across ranks, on CPU with gloo (world size 2)."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    import bench
    ws, r, local = bench.dist_env()
    assert (ws, r, local) == (world, rank, rank)
    # each replica reports its own device time and converged pairs
    ms, pairs = bench.combine_ranks(1000.0 * (rank + 1), 112 - rank, torch.device('cpu'))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ms, pairs))


def test_replicas_take_max_time_and_sum_pairs():
    import torch.multiprocessing as mp
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get() for _ in range(2))
    for rank, ms, pairs in out:
        assert ms == 2000.0            # max over ranks
        assert pairs == 112 + 111      # sum over ranks
