"""The N > 1 bench path on CPU ranks (gloo, world size 2): replicas integrate independent sweeps, the whole-job time
is the slowest rank's and the units add up."""
from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    t, n = bench.reduce_over_ranks(1.0 + rank, 100 * (rank + 1), dist, device="cpu")
    out[rank] = (t, n, bench.replica_seed("config2-block", rank))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_reduce_over_two_gloo_ranks():
    port = _free_port()
    manager = mp.get_context("spawn").Manager()     # no fork of a process that runs threads
    out = manager.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, start_method="spawn")
    assert out[0][:2] == (2.0, 300) and out[1][:2] == (2.0, 300)
    assert out[0][2] != out[1][2]
