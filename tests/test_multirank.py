"""The N > 1 path of bench.py: independent replicas, the job time is the slowest rank's
and the whole-job throughput counts every rank's evaluations. Run as two gloo ranks on
the CPU (the GPU runs of this build have one GPU)."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = 100.0 + 50.0 * rank          # rank 1 is the slow replica
        t = bench.max_over_ranks(local_ms, dist, "cpu")
        dist.barrier()
        out[rank] = (t, bench.replica_throughput(world, 20, t))
    finally:
        dist.destroy_process_group()


def test_replicas_report_the_slowest_rank_and_the_whole_job_throughput():
    world = 2
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as manager:
        out = manager.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    t, value = res[0]
    assert t == 150.0
    assert value == pytest.approx(world * 20 / 0.150)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(12.5, None, "cpu") == 12.5
    assert bench.replica_throughput(1, 10, 100.0) == pytest.approx(100.0)
