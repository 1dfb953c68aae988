"""Multi-process path of bench.py on CPU: two gloo ranks (the replicas form of --gpus N) agree
on the slowest rank's time and on the whole-job throughput."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    mine = 10.0 + 5.0 * rank  # per-rank timed milliseconds
    slowest = bench.max_over_ranks(mine, "cpu")
    out[rank] = (slowest, bench.whole_job_qps(1000, 4, world, slowest))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_and_throughput():
    world = 2
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn")
    assert out[0] == out[1]
    slowest, qps = out[0]
    assert slowest == 15.0
    assert qps == pytest.approx(world * 1000 * 4 / 0.015)


def test_single_process_is_its_own_max():
    import bench
    assert bench.max_over_ranks(3.5, "cpu") == 3.5
    assert bench.whole_job_qps(10000, 1, 1, 2.0) == pytest.approx(5e6)
