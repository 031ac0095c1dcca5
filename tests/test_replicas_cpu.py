"""The replica plumbing of bench.py with two processes on the host (gloo):
each rank times its own searches; the job time is the max over ranks and the
throughput the sum of what all ranks processed over that time."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench

    w, r, local, dist = bench.dist_setup(timeout_s=60)
    try:
        assert (w, r, local) == (world, rank, rank) and dist.get_backend() == "gloo"
        times = [0.010 * (rank + 1), 0.020 * (rank + 1)]       # seconds per step
        edges = [1e9, 1e9]                                      # traversed edges per step
        total = bench.barrier_max(dist, sum(times))
        done = bench.barrier_sum(dist, sum(edges))
        out[rank] = (total, done)
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_time_sum_work():
    import torch.multiprocessing as mp

    world = 2
    port = _free_port()
    # spawn throughout: no fork of a process that may hold threads
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    # every rank sees the slowest rank's time and the work of both
    for rank in range(world):
        total, done = res[rank]
        assert total == pytest.approx(0.060)
        assert done == pytest.approx(4e9)


def test_single_process_needs_no_group():
    import bench

    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    world, rank, local, dist = bench.dist_setup()
    assert (world, rank, local, dist) == (1, 0, 0, None)
    assert bench.barrier_max(None, 1.5) == 1.5 and bench.barrier_sum(None, 2.0) == 2.0
