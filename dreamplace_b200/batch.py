"""Batched global placement of many independent designs on one GPU.

Each design keeps its own GP loop (``NonLinearPlace.run_gen``), its own CUDA
stream and its own captured trial graphs.  The driver resumes the designs in
turn: a design's loop runs until it has enqueued its next trial on its stream
and yields, so up to one trial per design is in flight at a time and the
small-design kernels of different designs overlap on the GPU, while the host
reads each design's metrics only after the other designs have been enqueued.

Across GPUs the designs are partitioned (design i goes to rank i mod world);
ranks exchange nothing but their results at the end.

Usage: python -m dreamplace_b200.batch [--designs 64] [--seed 1] [--sequential]
  [--max-iterations N] [--repeat 2]; prints one JSON line (designs/s,
  per-design iteration latency p50 / p99 of the last batched pass, the first
  pass's time, and the same for the sequential loop with --sequential).
"""
import argparse
import json
import math
import os
import time

import numpy as np
import torch

from . import synthetic
from .nonlinear_place import NonLinearPlace
from .params import Params


def bins_for(num_cells, lo=64, hi=512):
    """Power of two nearest sqrt(cells), clamped to [lo, hi]."""
    return int(min(max(2 ** round(math.log2(math.sqrt(num_cells))), lo), hi))


def batch_set(count=64, seed=1, lo=5000, hi=200000):
    """Designs with movable counts log-uniform in [lo, hi], per-design seeds."""
    rng = np.random.RandomState(seed)
    counts = np.exp(rng.uniform(np.log(lo), np.log(hi), size=count)).astype(np.int64)
    return [synthetic.scaled(int(c), num_bins=bins_for(int(c)), seed=seed * 1000 + i, name="batch%d" % i)
            for i, c in enumerate(counts)]


def assign(num_designs, rank, world):
    """Designs handled by `rank` of `world` (round robin)."""
    return list(range(rank, num_designs, world))


def params_for(design, deterministic=0):
    return Params(target_density=design.target_density, stop_overflow=0.07, dct_precision="split_bf16",
                  deterministic_flag=deterministic)


class BatchPlacer(object):
    """Global placement of a list of designs, interleaved on one device."""

    def __init__(self, designs, device="cuda", deterministic=0):
        self.designs = designs
        self.placers = [NonLinearPlace(params_for(d, deterministic), d, device) for d in designs]

    def run(self, max_iterations=None):
        """All designs to completion.  Returns (results, per-iteration latencies in s)."""
        n = len(self.designs)
        streams = [torch.cuda.Stream() for _ in range(n)]
        gens = [pl.run_gen(pl.params, d, max_iterations) for pl, d in zip(self.placers, self.designs)]
        results = [None] * n
        latencies = []
        last = [None] * n
        active = list(range(n))
        home = torch.cuda.current_stream()
        try:
            while active:
                still = []
                for i in active:
                    # set_stream, not a stream context: the context's current-stream
                    # lookups cost more host time than a small design's iteration
                    torch.cuda.set_stream(streams[i])
                    try:
                        next(gens[i])
                        now = time.perf_counter()
                        if last[i] is not None:
                            latencies.append(now - last[i])
                        last[i] = now
                        still.append(i)
                    except StopIteration as stop:
                        results[i] = stop.value
                active = still
        finally:
            torch.cuda.set_stream(home)
        torch.cuda.synchronize()
        return results, latencies

    def run_sequential(self, max_iterations=None):
        """The single-design path in a loop, for comparison."""
        results, latencies = [], []
        for pl, d in zip(self.placers, self.designs):
            results.append(pl(pl.params, d, max_iterations=max_iterations))
            latencies.extend(pl.iteration_times)
        torch.cuda.synchronize()
        return results, latencies


def summary(label, designs, results, latencies, seconds):
    """designs/s, per-design iteration latency p50 / p99, iterations and the
    mean final overflow of one pass; a rank without designs reports zeros
    (and no overflow)."""
    if not designs:
        return {label + "_designs_per_s": 0.0, label + "_seconds": 0.0, label + "_iteration_ms_p50": 0.0,
                label + "_iteration_ms_p99": 0.0, label + "_iterations": 0, label + "_mean_final_overflow": None}
    lat = np.array(latencies) * 1000.0 if latencies else np.zeros(1)
    finals = [r[-1][-1][-1] for r in results]
    return {label + "_designs_per_s": round(len(designs) / seconds, 3) if seconds > 0 else 0.0,
            label + "_seconds": round(seconds, 3),
            label + "_iteration_ms_p50": round(float(np.percentile(lat, 50)), 3),
            label + "_iteration_ms_p99": round(float(np.percentile(lat, 99)), 3),
            label + "_iterations": int(sum(f.iteration + 1 for f in finals)),
            label + "_mean_final_overflow": round(float(np.mean([f.overflow for f in finals])), 4)}


def place_partition(designs_all, rank, world, run_pass, repeat=1):
    """The designs of this rank (round robin), placed by run_pass(designs) ->
    (results, latencies) `repeat` times; the last pass is summarised (the
    first also pays the process's one-time costs and is reported apart).  A
    rank without designs places nothing and reports zeros."""
    mine = [designs_all[i] for i in assign(len(designs_all), rank, world)]
    out = {"designs": len(designs_all), "designs_on_rank": len(mine), "world": world,
           "cells": int(sum(d.num_movable_nodes for d in mine))}
    res, lat, seconds = [], [], 0.0
    if mine:
        for r in range(max(repeat, 1)):
            t0 = time.perf_counter()
            res, lat = run_pass(mine)
            seconds = time.perf_counter() - t0
            if r == 0 and repeat > 1:
                out["batched_first_pass_seconds"] = round(seconds, 3)
                out["batched_first_pass_designs_per_s"] = round(len(mine) / seconds, 3)
    out.update(summary("batched", mine, res, lat, seconds))
    return out


def gather_partition(out, rank, world, num_designs):
    """Every rank's summary to rank 0 (one all_gather_object, the only
    collective); rank 0 reports designs/s of the whole job, timed by the
    slowest rank.  Returns the combined summary on rank 0, this rank's
    otherwise."""
    if world == 1:
        return out
    import torch.distributed as dist
    gathered = [None] * world
    dist.all_gather_object(gathered, out)
    if rank != 0:
        return out
    secs = max(g["batched_seconds"] for g in gathered)
    return {"designs": num_designs, "world": world,
            "batched_designs_per_s": round(num_designs / secs, 3) if secs > 0 else 0.0,
            "slowest_rank_seconds": secs, "per_rank": gathered}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--designs", type=int, default=64)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--max-iterations", type=int, default=None)
    ap.add_argument("--sequential", action="store_true", help="also time the single-design loop")
    ap.add_argument("--repeat", type=int, default=2,
                    help="batched passes over the same designs; the last one is reported (the first also "
                         "pays the process's one-time set-up, reported as batched_first_pass_*)")
    ap.add_argument("--backend", default="nccl", choices=["nccl", "gloo"],
                    help="process-group backend for the final exchange of results (multi-rank runs)")
    args = ap.parse_args(argv)
    if not torch.cuda.is_available():
        raise SystemExit("batch placement needs a CUDA device")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group(args.backend, timeout=datetime.timedelta(seconds=600))
    designs_all = batch_set(args.designs, args.seed)

    def run_pass(designs):
        # each pass places the same designs with new placers, as a service
        # placing batch after batch would
        bp = BatchPlacer(designs)
        torch.cuda.synchronize()
        res, lat = bp.run(args.max_iterations)
        del bp
        return res, lat

    out = place_partition(designs_all, rank, world, run_pass, args.repeat)
    mine = [designs_all[i] for i in assign(len(designs_all), rank, world)]
    if args.sequential and mine:
        seq = BatchPlacer(mine)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res, lat = seq.run_sequential(args.max_iterations)
        out.update(summary("sequential", mine, res, lat, time.perf_counter() - t0))
    out = gather_partition(out, rank, world, len(designs_all))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
