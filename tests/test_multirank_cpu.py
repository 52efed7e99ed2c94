"""Multi-process plumbing of bench.py on CPU with gloo, world size 2.

The detector shards by image (replicas): ranks never exchange data; the only
collectives are the barrier and the max over ranks of the timed region.
"""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, results):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 10.0 + 5.0 * rank          # rank 1 is the slow one
        m = bench.max_over_ranks(local_ms, world)
        dist.barrier()
        v = bench.replica_throughput(1920 * 1080, 100, world, m)
        results[rank] = (m, v)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_throughput_gloo():
    import torch.multiprocessing as mp
    world = 2
    mgr = mp.get_context("spawn").Manager()
    results = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), results), nprocs=world, start_method="spawn", join=True)
    assert results[0][0] == results[1][0] == 15.0
    # whole-job throughput: both ranks' pixels over the slowest rank's time
    expect = 2 * 100 * 1920 * 1080 / 15e-3 / 1e6
    assert results[0][1] == pytest.approx(expect) and results[1][1] == pytest.approx(expect)


def test_single_rank_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_throughput(100, 10, 1, 1.0) == pytest.approx(1.0)


def test_reference_arm_other_ranks_do_no_work(capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    class A:
        steps = 1
        warmup = 1
    bench.run_reference(A(), rank=1, world=2)
    assert capsys.readouterr().out == ""
