"""Multi-GPU runs are independent replicas (one simulation does not shard):
bench.py's whole-job throughput is the units of all ranks over the slowest
rank's time.  Checked with two gloo ranks on the CPU."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, results):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        ms = [100.0, 250.0][rank]  # the second rank is the slow one
        units = [1000, 1000][rank]
        value, ms_max = bench.replica_throughput(ms, units, dist)
        results[rank] = (value, ms_max)
    finally:
        dist.destroy_process_group()


def test_two_replicas_use_max_time_and_sum_of_units():
    port = 29500 + os.getpid() % 1000
    with mp.get_context("spawn").Manager() as m:
        results = m.dict()
        mp.start_processes(_rank, args=(2, port, results), nprocs=2, join=True, start_method="spawn")
        res = dict(results)
    for rank in (0, 1):
        value, ms_max = res[rank]
        assert ms_max == pytest.approx(250.0)
        assert value == pytest.approx(2000 / 0.25)


def test_single_rank_without_a_group():
    sys.path.insert(0, ROOT)
    import bench

    value, ms_max = bench.replica_throughput(50.0, 500)
    assert ms_max == 50.0 and value == pytest.approx(10000.0)
