"""The bench's replica timing across ranks (barrier, max time, summed hits),
on CPU with gloo, world size 2."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    t_local = 1.0 + rank          # rank 1 is the slow one
    hits = 100.0 * (rank + 1)
    t_max, hits_all = bench.reduce_over_ranks(t_local, hits, dist, torch.device("cpu"))
    out[rank] = (t_max, hits_all)
    dist.barrier()
    dist.destroy_process_group()


def test_replica_reduction():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn")
        for r in range(world):
            t_max, hits_all = out[r]
            assert t_max == 2.0
            assert hits_all == 300.0
