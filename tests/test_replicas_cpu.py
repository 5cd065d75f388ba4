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


def test_clock_summary():
    """bench.py's clock record from nvidia-smi rows: the median SM clock under load, the
    max clock, and only the throttle reasons reported Active ("Not Active" is not one)."""
    import sys

    sys.path.insert(0, REPO)
    import bench

    rows = ["0, 1965, 1965, 700.1 , 0x0000000000000000, Not Active, Not Active, Not Active, Not Active\n",
            "0, 1800, 1965, 990.5 , 0x0000000000000004, Not Active, Not Active, Not Active, Active\n",
            "0, 1900, 1965, 950.0 , 0x0000000000000004, Not Active, Not Active, Not Active, Active\n",
            "[N/A], [N/A], [N/A], [N/A], [N/A], [N/A], [N/A], [N/A], [N/A]\n", "garbage\n"]
    out = bench.summarize_clocks(rows)
    assert out == {"sm_mhz": 1900.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    assert bench.summarize_clocks([]) is None
