"""The bench's replica plumbing (one process per GPU, host-side gloo barrier and
max/sum reductions of timings and counts) with two ranks on the CPU."""

import os
import socket

import torch.multiprocessing as mp

from conftest import REPO


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, REPO)
    import bench

    d = bench.Dist(world)
    d.barrier()
    out[rank] = (d.max(1.5 + rank), d.sum(10.0 * (rank + 1)))
    d.barrier()
    d.close()


def test_two_replicas_reduce_over_gloo():
    world = 2
    out = mp.get_context("spawn").Manager().dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    for r in range(world):
        assert out[r] == (2.5, 30.0)  # max over ranks of 1.5 + rank; sum of 10, 20


def test_single_process_needs_no_group():
    import sys

    sys.path.insert(0, REPO)
    import bench

    d = bench.Dist(1)
    assert d.max(3.0) == 3.0 and d.sum(4.0) == 4.0
    d.barrier()
    d.close()
