"""Field maps stored vs recomputed in backward: peak HBM and iterations/s.

A 1M-movable-cell design at 1024x1024 bins (same generator and ratios as the
2.1M-cell design: 1.05M nets, 476 macros, 70% utilisation) runs a fixed number of GP
iterations on

* the reference-shaped autograd path (``gp_engine="autograd"``) with the
  electric potential's field maps stored between forward and backward
  (``recompute_field=0``, the reference's behaviour,
  dreamplace/ops/electric_potential/electric_potential.py:200-217) and
  recomputed in backward (``recompute_field=1``);
* the graph-captured engine, for comparison (its buffers are allocated once,
  so it has no stored/recomputed distinction).

For each: the peak device memory of the whole run (torch caching allocator,
``max_memory_allocated``) and of the steady-state iterations alone (the peak
after iteration ``--warmup`` minus what was allocated then), and iterations/s
over the iterations after the warm-up (host wall clock between iteration
ends; each iteration ends with a device-to-host read of its metrics, so the
wall clock covers the device work).

Usage: python -m dreamplace_b200.memory_study [--cells 1000000] [--bins 1024]
  [--iterations 200] [--warmup 20] [--precision split_bf16] [--variant NAME]
Prints one JSON line per variant (each variant runs in a fresh process).
"""
import argparse
import json
import subprocess
import sys
import time

import torch

from . import synthetic
from .nonlinear_place import place
from .params import Params


VARIANTS = {"autograd-stored": ("autograd", False), "autograd-recomputed": ("autograd", True),
            "graph": ("graph", False)}


def run_variant(design, engine, recompute, iterations, warmup, precision):
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    torch.cuda.reset_peak_memory_stats()
    start_alloc = torch.cuda.memory_allocated()
    marks = {}

    def callback(it, _metrics):
        if it == warmup - 1:
            torch.cuda.synchronize()
            marks["alloc"] = torch.cuda.memory_allocated()
            marks["run_peak"] = torch.cuda.max_memory_allocated()
            torch.cuda.reset_peak_memory_stats()
            marks["t0"] = time.perf_counter()
        if it == iterations - 1:
            torch.cuda.synchronize()
            marks["t1"] = time.perf_counter()

    # stop_overflow 0 keeps every variant running the same number of iterations
    p = Params(target_density=design.target_density, stop_overflow=0.0, dct_precision=precision,
               gp_engine=engine, recompute_field=int(recompute))
    placer, res = place(design, p, max_iterations=iterations, callback=callback)
    torch.cuda.synchronize()
    steady_peak = torch.cuda.max_memory_allocated()
    n = res["iterations"] - warmup
    line = {"engine": engine, "field": "recomputed" if recompute else "stored", "precision": precision,
            "cells": design.num_movable_nodes, "bins": design.num_bins_x, "iterations_timed": n,
            "iters_per_s": round(n / (marks["t1"] - marks["t0"]), 2),
            "run_peak_mib": round((max(marks["run_peak"], steady_peak) - start_alloc) / 2 ** 20, 1),
            "steady_peak_mib": round(steady_peak / 2 ** 20, 1),
            "steady_transient_mib": round((steady_peak - marks["alloc"]) / 2 ** 20, 1),
            "hpwl": res["hpwl"], "overflow": res["overflow"]}
    del placer
    return line


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--cells", type=int, default=1_000_000)
    ap.add_argument("--bins", type=int, default=1024)
    ap.add_argument("--iterations", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--precision", default="split_bf16")
    ap.add_argument("--variant", choices=sorted(VARIANTS), default=None, help="run one variant in this process")
    args = ap.parse_args(argv)
    if not torch.cuda.is_available():
        raise SystemExit("memory_study needs a CUDA device")
    if args.variant is None:
        # each variant in a process of its own, so that no variant's cached
        # allocations or transform matrices count toward another's peak
        for v in VARIANTS:
            subprocess.run([sys.executable, "-m", "dreamplace_b200.memory_study", "--variant", v,
                            "--cells", str(args.cells), "--bins", str(args.bins), "--iterations",
                            str(args.iterations), "--warmup", str(args.warmup), "--precision", args.precision],
                           check=True)
        return 0
    engine, recompute = VARIANTS[args.variant]
    design = synthetic.scaled(args.cells, num_bins=args.bins, seed=1, name="gp%dk" % (args.cells // 1000))
    print(json.dumps(run_variant(design, engine, recompute, args.iterations, args.warmup, args.precision)),
          flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
