"""The multi-GPU path of bench.py is N independent replicas; its only exchange is the
max-over-ranks reduction of the timed legs. Checked here with two gloo ranks on CPU."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r took (r + 1) x the time of rank 0 on every leg
        ms = [10.0 * (rank + 1), 20.0 * (rank + 1), 40.0 * (rank + 1)]
        mx, rates = bench.job_rates(torch, ms, [20, 5, 20], world, dist, "cpu")
        q.put((rank, mx, rates))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, rates in got:
        assert mx == pytest.approx([20.0, 40.0, 80.0])  # the slowest rank's times
        # whole-job rate: all ranks' units over the slowest time
        assert rates == pytest.approx([2 * 20 / 0.020, 2 * 5 / 0.040, 2 * 20 / 0.080])


def test_single_rank_rate():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    mx, rates = bench.job_rates(torch, [8.5], [10], 1)
    assert mx == [8.5] and rates == pytest.approx([10 / 0.0085])
