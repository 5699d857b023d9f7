"""The multi-GPU path is replicas only: each rank runs an independent copy of the workload
and bench.py reports all ranks' terms over the slowest rank's time.  The aggregation runs
here as two gloo ranks on the CPU (no GPU involved)."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        terms = [3.0e9, 5.0e9][rank]
        ms = [800.0, 1000.0][rank]
        value, max_ms, all_terms = bench.replica_throughput(terms, ms, world)
        out[rank] = (value, max_ms, all_terms)
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_replica_throughput_is_total_terms_over_slowest_rank():
    world = 2
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
    for rank in range(world):
        value, max_ms, all_terms = out[rank]
        assert max_ms == 1000.0
        assert all_terms == 8.0e9
        assert value == pytest.approx(8.0e9 / 1.0)
