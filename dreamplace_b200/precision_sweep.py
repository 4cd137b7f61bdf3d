"""Precision sweep of the Poisson solve.

For transform sizes 512^2 .. 4096^2 and each solve precision (fp32, tf32,
bf16, split-bf16) this measures

* the error of the field maps (max-norm relative) and of the energy against an
  fp64 evaluation of the same matrix forms (the reference's dct2_fft2 /
  idxst_idct / idct_idxst / idct2 scalings, electric_potential.py:504-519),
* the device time of one solve (CUDA events over graph replays) and the GEMM
  throughput it implies,

on density maps rasterised from the 10k-cell design's GP positions at
iterations 0, 300 and 700; and with ``--gp`` the end-of-GP HPWL, overflow and
iteration count of that design for each precision.

Usage: python -m dreamplace_b200.precision_sweep [--sizes 512,1024,2048,4096] [--gp]
Prints one JSON object per line.
"""
import argparse
import json
import math

import numpy as np
import torch

from . import synthetic
from ._native import C, precision_code
from .dct2_fft2 import cos_matrix, icos_matrix, isin_matrix
from .electric_potential import poisson_flops, poisson_solve
from .nonlinear_place import place
from .params import Params

PRECISIONS = ("fp32", "tf32", "bf16", "split_bf16")


def snapshots(design, iterations):
    """GP positions of the design after each number of iterations (deterministic runs)."""
    out = {}
    for it in iterations:
        p = Params(target_density=design.target_density, stop_overflow=0.07, dct_precision="fp32",
                   deterministic_flag=1)
        placer, res = place(design, p, max_iterations=max(it, 1))
        out[it] = (placer.pos[0].detach().clone(), res["iterations"])
    return out


def density_on_grid(design, pos, M):
    """Triangle-model density map of movable + filler cells on an M x M grid over the die."""
    dev = pos.device
    bs = (design.xh - design.xl) / M
    sx = torch.from_numpy(design.node_size_x).to(dev)
    sy = torch.from_numpy(design.node_size_y).to(dev)
    sxc = sx.clamp(min=bs * math.sqrt(2))
    syc = sy.clamp(min=bs * math.sqrt(2))
    ox, oy = (sx - sxc).mul(0.5), (sy - syc).mul(0.5)
    ratio = sx * sy / (sxc * syc)
    init = torch.zeros(M * M, device=dev)
    dmap = C.density_map(pos, sxc, syc, ox, oy, ratio, init, init, init, 1.0, design.xl, design.yl, design.xh,
                         design.yh, bs, bs, design.num_movable_nodes, design.num_filler_nodes, 0, M, M, 0, 0, 0, 0,
                         0, None)
    return dmap.view(M, M), bs


def fp64_solve(rho, bs):
    """(Ex, Ey, energy) of a normalised density map in fp64 (same matrix forms)."""
    dev = rho.device
    M, N = rho.shape
    t = lambda a: torch.from_numpy(a).to(dev)  # noqa: E731
    cM, cN = t(cos_matrix(M)), t(cos_matrix(N))
    chM, chN, shM, shN = t(icos_matrix(M)), t(icos_matrix(N)), t(isin_matrix(M)), t(isin_matrix(N))
    r = rho.double()
    a = 4.0 / (M * N) * (cM @ r @ cN.T)
    wu = (torch.arange(M, dtype=torch.float64, device=dev) * (2 * math.pi / M))[:, None]
    wv = (torch.arange(N, dtype=torch.float64, device=dev) * (2 * math.pi / N))[None, :]
    d = wu * wu + wv * wv
    d[0, 0] = 1.0
    inv = 1.0 / d
    inv[0, 0] = 0.0
    ex = 4.0 * (shM @ (a * wu * inv / 2) @ chN.T)
    ey = 4.0 * (chM @ (a * wv * inv / 2) @ shN.T)
    phi = 4.0 * (chM @ (a * inv) @ chN.T)
    return ex, ey, float((phi * r).sum())


def graph_ms(fn, reps=10):
    fn()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    g.replay()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        g.replay()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def sweep_sizes(design, snaps, sizes):
    for M in sizes:
        for it, (pos, _) in snaps.items():
            dmap, bs = density_on_grid(design, pos, M)
            rho = (dmap / (bs * bs)).contiguous()
            rex, rey, renergy = fp64_solve(rho, bs)
            for prec in PRECISIONS:
                ex, ey, energy = poisson_solve(rho, bs, bs, prec)
                err = max(float((ex.double() - rex).abs().max() / rex.abs().max()),
                          float((ey.double() - rey).abs().max() / rey.abs().max()))
                line = {"size": M, "gp_iteration": it, "precision": prec, "field_rel_err": err,
                        "energy_rel_err": abs(float(energy.item()) - renergy) / abs(renergy)}
                if it == min(snaps):
                    ms = graph_ms(lambda: poisson_solve(rho, bs, bs, prec))
                    line.update(solve_ms=round(ms, 4),
                                gemm_tflops=round(poisson_flops(M, M, prec) / (ms * 1e-3) / 1e12, 1))
                print(json.dumps(line), flush=True)
            del rex, rey
            torch.cuda.empty_cache()


def sweep_gp(design):
    for prec in PRECISIONS:
        p = Params(target_density=design.target_density, stop_overflow=0.07, dct_precision=prec,
                   deterministic_flag=1)
        _, res = place(design, p)
        print(json.dumps({"design": design.name, "precision": prec, "iterations": res["iterations"],
                          "hpwl": res["hpwl"], "overflow": res["overflow"]}), flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--sizes", default="512,1024,2048,4096")
    ap.add_argument("--iterations", default="0,300,700")
    ap.add_argument("--gp", action="store_true", help="also run the full GP per precision")
    args = ap.parse_args(argv)
    if not torch.cuda.is_available():
        raise SystemExit("precision_sweep needs a CUDA device")
    precision_code("split_bf16")
    design = synthetic.cells_10k()
    snaps = snapshots(design, [int(x) for x in args.iterations.split(",")])
    sweep_sizes(design, snaps, [int(x) for x in args.sizes.split(",")])
    if args.gp:
        sweep_gp(design)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
