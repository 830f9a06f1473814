"""Replicas on CPU with the gloo backend (world size 2): the job's throughput is all ranks'
samples over the slowest rank's time; no rank's work depends on another's."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from hypertrace_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        samples = 1000.0 * (rank + 1)
        seconds = 0.5 + rank
        tot, mx, hops = replicas.aggregate(samples, seconds, hops=10.0 * (rank + 1))
        out[rank] = (tot, mx, hops, replicas.replica_seed(123, rank))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    for r in range(world):
        tot, mx, hops, seed = out[r]
        assert tot == 3000.0 and mx == 1.5 and hops == 30.0
    assert out[0][3] != out[1][3]


def test_single_process_identity():
    assert replicas.aggregate(5.0, 2.0, 7.0) == (5.0, 2.0, 7.0)
