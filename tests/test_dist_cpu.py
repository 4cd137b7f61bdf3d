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


class _Stub(object):
    """A design stand-in: the partition only reads the movable-cell count."""

    def __init__(self, i):
        self.name = "stub%d" % i
        self.num_movable_nodes = 1000 * (i + 1)


class _Metric(object):
    def __init__(self, it, overflow):
        self.iteration = it
        self.overflow = overflow


def _batch_worker(rank, world, port, num_designs, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from dreamplace_b200 import batch
    designs = [_Stub(i) for i in range(num_designs)]
    placed = []

    def run_pass(ds):
        # a CPU stand-in for the GPU placer: one GP "iteration" per design,
        # slower on rank 1 so the job is timed by it
        placed.extend(d.name for d in ds)
        import time
        time.sleep(0.05 * (rank + 1))
        return [[[[_Metric(9, 0.06)]]] for _ in ds], [0.001] * len(ds)

    summ = batch.place_partition(designs, rank, world, run_pass)
    res = batch.gather_partition(summ, rank, world, num_designs)
    out[rank] = len(placed)
    if rank == 0:
        out[world] = res["batched_designs_per_s"]
        out[world + 1] = res["slowest_rank_seconds"]
        out[world + 2] = sum(g["designs_on_rank"] for g in res["per_rank"])
        out[world + 3] = float(all(g["batched_mean_final_overflow"] in (None, 0.06) for g in res["per_rank"]))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("num_designs", [3, 1])
def test_two_rank_batch_partition_and_gather(num_designs):
    """dreamplace_b200.batch across two gloo ranks with CPU stand-in placers:
    round-robin partition (rank 0 gets designs 0, 2, rank 1 design 1; with a
    single design rank 1 gets none and reports zeros), the one all_gather of
    the results, and designs/s of the whole job timed by the slowest rank."""
    world = 2
    out = torch.zeros(world + 4, dtype=torch.float64).share_memory_()
    mp.spawn(_batch_worker, args=(world, _free_port(), num_designs, out), nprocs=world, join=True)
    per_rank = [len(range(r, num_designs, world)) for r in range(world)]
    assert [int(out[r]) for r in range(world)] == per_rank
    assert int(out[world + 2]) == num_designs
    slowest = float(out[world + 1])
    assert slowest > 0
    assert out[world] == pytest.approx(round(num_designs / slowest, 3), rel=1e-3)
    assert out[world + 3] == 1.0
