"""bench.py's multi-GPU form is replicas only (each rank solves its own problem; no data-path
collective): the job time is the slowest rank's, the value counts every rank's DOFs, and ranks start
on different k fields. Checked here with two gloo ranks on the CPU."""

import os
import socket
import sys
from datetime import timedelta

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench

    ms = bench.max_over_ranks(10.0 + 5.0 * rank, world)
    fields = [bench.replica_field(i, rank) for i in range(4)]
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, ms, fields))


def test_two_gloo_ranks_time_is_the_slowest_and_problems_differ():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    try:
        for _ in range(2):
            rank, ms, fields = out.get(timeout=120)
            res[rank] = (ms, fields)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert res[0][0] == res[1][0] == 15.0  # max over ranks
    assert res[0][1] != res[1][1]  # rank r starts at field r
    assert res[1][1][0] == 1 and res[0][1][0] == 0


def test_whole_job_value_counts_every_rank():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.whole_job_value(1000, 4, 2.0) == pytest.approx(4 * 1000 / 2e-3)
    assert bench.max_over_ranks(3.5, 1) == 3.5
