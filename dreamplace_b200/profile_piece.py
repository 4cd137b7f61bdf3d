"""One piece of the GP trial on a GP state, for single-launch profiler captures.

    python -m dreamplace_b200.profile_piece --piece wa --iterations 1499

Runs global placement of a synthetic design (graph engine, split-BF16 Poisson
solve, fp32 scatter) to the given iteration, refreshes the visiting order at
the position reached, then runs the chosen piece ``--repeat`` times on it with
a synchronize after each run, inside the NVTX range ``profile_piece``.  Under
ncu, ``--nvtx --nvtx-include "profile_piece/" -k <kernel> -s 1 -c 1`` then
captures one warm launch of the piece's kernel.  Pieces:

* ``wa``: WA forward + HPWL (``wa_lane_kernel``);
* ``scatter``: the split density scatter (``tile_scatter_kernel``,
  ``finish_maps_kernel``);
* ``poisson``: the Poisson solve of the current density map (``tc_gemm_kernel``);
* ``field``: the field gather (``electric_force_records_kernel``);
* ``assemble``: gradient assembly + preconditioner (``assemble_precondition_kernel``);
* ``trial``: the Nesterov trial point (``nesterov_trial_kernel``).
"""
import argparse

import torch

from . import synthetic
from .electric_potential import poisson_solve
from .nonlinear_place import NonLinearPlace
from .params import Params

PIECES = ("wa", "scatter", "poisson", "field", "assemble", "trial")


def run_piece(eng, piece, repeat):
    ep = eng.ep
    p = eng.slot
    q = eng.next_slot(p)
    v, g = eng.V[p], eng.G[p]
    vn, gn = eng.V[q], eng.G[q]
    saved = eng.S[p].clone()
    eng.scatter_maps(v, eng.O[q])
    rho = eng.dmap.mul(1.0 / (ep.bin_size_x * ep.bin_size_y))
    ex, ey, _ = poisson_solve(rho, ep.bin_size_x, ep.bin_size_y, eng.prec)
    torch.cuda.synchronize()
    # the piece's launches sit in the NVTX range "profile_piece" (ncu --nvtx
    # --nvtx-include "profile_piece/" captures them and none of the GP run's)
    torch.cuda.nvtx.range_push("profile_piece")
    for _ in range(repeat):
        if piece == "wa":
            eng.wirelength(v, eng.H[q])
        elif piece == "scatter":
            eng.scatter_maps(v, eng.O[q])
        elif piece == "poisson":
            poisson_solve(rho, ep.bin_size_x, ep.bin_size_y, eng.prec)
        elif piece == "field":
            eng.field_force(v, ex, ey)
        elif piece == "assemble":
            eng.assemble(v, g, vn, gn)
        elif piece == "trial":
            eng.nesterov_trial_only(p)
        torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    eng.S[p].copy_(saved)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--piece", choices=PIECES, required=True)
    ap.add_argument("--design", default="cells_2m", choices=["cells_10k", "cells_2m"])
    ap.add_argument("--iterations", type=int, default=1499, help="GP iterations run before the piece")
    ap.add_argument("--repeat", type=int, default=2)
    args = ap.parse_args(argv)
    design = synthetic.cells_2m() if args.design == "cells_2m" else synthetic.cells_10k()
    params = Params(target_density=design.target_density, stop_overflow=0.0, dct_precision="split_bf16",
                    deterministic_flag=0)
    placer = NonLinearPlace(params, design, "cuda")
    placer(params, design, max_iterations=args.iterations)
    eng = placer.stepper.eng
    torch.cuda.synchronize()
    eng.refresh_order(eng.current_position())
    run_piece(eng, args.piece, args.repeat)
    print("ran %s %d times at iteration %d" % (args.piece, args.repeat, args.iterations))


if __name__ == "__main__":
    main()
