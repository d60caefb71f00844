"""The multi-GPU path of bench.py (replicas, one process per GPU) on the CPU:
two gloo ranks, barrier, max-over-ranks timing and whole-job throughput."""

import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from ddhdg_b200 import replicas

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        replicas.barrier()
        ms = 10.0 + 5.0 * rank            # the ranks' own timings
        slow = replicas.max_over_ranks(ms, "cpu")
        out.put((rank, replicas.world_size(), slow, replicas.job_throughput(1000, slow)))
        replicas.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, world, slow, thr in res:
        assert world == 2
        assert slow == 15.0                          # max over the ranks
        assert thr == pytest.approx(2 * 1000 / 15e-3)  # all ranks' units / slowest time


def test_single_process_is_its_own_job():
    from ddhdg_b200 import replicas

    assert replicas.world_size() == 1
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.job_throughput(100, 2.0) == pytest.approx(5e4)
