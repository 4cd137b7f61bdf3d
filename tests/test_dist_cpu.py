"""The multi-GPU bench path on CPU: two gloo ranks run the barrier and
max-over-ranks timing helpers bench.py uses with NCCL, and the replica
aggregation (one design per rank, no data-path collective)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    bench.barrier(world)
    ms = 100.0 + 50.0 * rank  # rank 1 is the slowest
    m = bench.max_over_ranks(ms, world, device="cpu")
    out[rank] = m
    out[world + rank] = bench.replica_value(30, world, m)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_max_and_replica_value():
    world = 2
    out = torch.zeros(2 * world, dtype=torch.float64).share_memory_()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0] == out[1] == 150.0
    assert out[2] == out[3] == pytest.approx(2 * 30 / 0.150)
