#!/usr/bin/env python
"""Benchmark: global-placement iterations per second on the 2.1M-cell design.

Workload: the 2.1M-movable-cell synthetic design (1,000 macros, 2.2M nets,
~7.1M pins, ~0.99M fillers, 1024x1024 bins, 70% utilisation), seeded.  A
"step" is one GP iteration of the Nesterov loop (HPWL + overflow evaluation
and one optimizer step with >= 1 objective/gradient evaluation).  W untimed
warm-up iterations run first; then K iterations are timed with CUDA events
(barrier + synchronize on both sides, max over ranks).  The per-iteration
working set (pin arrays ~200 MB) exceeds the 126 MB L2, so no explicit flush
is done.

Arms:
  default            this implementation (split-BF16 Poisson solve unless
                     --precision), plus the plain fp32 form timed on the same
                     GPU for the headline comparison
  --impl reference   the reference's own CPU ops (built from the reference
                     sources into oracle/_ref) composed into the same GP
                     iteration, on all host cores

Multi-GPU (--gpus N under torchrun): one design per rank, replicas only (the
single-design path does not shard); value = iterations of all ranks / max time.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = "GP iters/s at 2.1M cells, plain FP32 vs split-BF16 DCT, at equal HPWL ±0.1%"
UNIT = "GP iter/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="split_bf16")
    ap.add_argument("--design", default="cells_2m", choices=["cells_10k", "cells_2m"])
    ap.add_argument("--no-plain", action="store_true", help="skip the plain fp32 comparison run")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-full-gp", action="store_true",
                    help="skip the runs of both Poisson-solve forms to the 0.07 overflow stop")
    ap.add_argument("--cpu-sample-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true", help="skip the host round-trip run (profiling)")
    ap.add_argument("--process-warmup", type=int, default=50,
                    help="GP iterations of an untimed run of the same design before the timed run (0: none)")
    ap.add_argument("--no-dropin", action="store_true",
                    help="skip timing the reference-facing modules (ElectricPotential, WeightedAverageWirelength)")
    ap.add_argument("--no-roofline", action="store_true", help="skip the per-kernel timing (profiling)")
    ap.add_argument("--skip-to", type=int, default=0,
                    help="run this many GP iterations untimed before the warm-up (times a later GP stage; "
                         "profiling)")
    ap.add_argument("--no-speculate", action="store_true",
                    help="enqueue each GP iteration after the host read the previous one (profiling: no trial is "
                         "enqueued ahead and voided)")
    return ap.parse_args()


def make_design(name):
    from dreamplace_b200 import synthetic
    return synthetic.cells_2m() if name == "cells_2m" else synthetic.cells_10k()


# ------------------------------------------------------------------ clocks
class ClockSampler(object):
    """nvidia-smi samples of SM clock and throttle reasons around the timed region.

    nvidia-smi is started, and its first sample awaited, before the GP warm-up:
    its start-up (NVML initialisation) can hold the driver for seconds and must
    not land inside the timed region.  Samples are stamped on arrival; the
    summary uses those that arrived between begin() and end() plus one
    sampling period after, or the nearest sample when the region is shorter
    than a period."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD_MS = 200

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.t_begin = self.t_end = None

    def start(self, ready_timeout=20.0):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", str(self.PERIOD_MS)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
            return
        t0 = time.time()
        while not self.lines and time.time() - t0 < ready_timeout and self.proc.poll() is None:
            time.sleep(0.02)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def begin(self):
        self.t_begin = time.time()

    def end(self):
        self.t_end = time.time()

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(1.5 * self.PERIOD_MS / 1000.0)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        parsed = []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for t, ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm, mx = float(p[1]), float(p[2])
            except ValueError:
                continue
            parsed.append((t, sm, mx, [nm for nm, v in zip(names, p[5:9]) if v.lower().startswith("active")]))
        if not parsed:
            return None
        tb = self.t_begin if self.t_begin is not None else parsed[0][0]
        te = (self.t_end if self.t_end is not None else parsed[-1][0]) + self.PERIOD_MS / 1000.0
        inside = [x for x in parsed if tb <= x[0] <= te]
        if not inside:
            inside = [min(parsed, key=lambda x: abs(x[0] - tb))]
        reasons = sorted({r for x in inside for r in x[3]})
        return {"sm_mhz": statistics.median(x[1] for x in inside), "sm_max_mhz": max(x[2] for x in inside),
                "reasons": reasons, "samples": len(inside)}


# ------------------------------------------------------------------ distributed
def dist_setup(gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, local, world


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v, world, device="cuda"):
    """Max of a per-rank float over all ranks (NCCL on the GPU path, gloo on CPU)."""
    if world == 1:
        return v
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(steps, world, ms_max):
    """Whole-job iterations/s of `world` independent replicas timed by the slowest rank."""
    return world * steps / (ms_max / 1000.0)


# ------------------------------------------------------------------ our arm
class TimedRun(object):
    """Runs the GP loop and times iterations [warmup, warmup + steps) with CUDA events."""

    def __init__(self, design, precision, world, e2e=False, time_pieces=False, speculate=True):
        from dreamplace_b200.nonlinear_place import NonLinearPlace
        from dreamplace_b200.params import Params
        self.params = Params(target_density=design.target_density, stop_overflow=0.07, dct_precision=precision,
                             deterministic_flag=0, time_pieces=time_pieces, speculate=speculate)
        self.dominant = None
        self.dominant_ms = None
        self.design = design
        self.world = world
        self.placer = NonLinearPlace(self.params, design, "cuda")
        self.e2e = e2e
        # the host round trip runs in E2E_CHUNKS pieces on two copy streams:
        # the upload of piece i overlaps the download of piece i + 1 (PCIe is
        # full duplex and each direction has its own copy engine)
        self.copy_streams = (torch.cuda.Stream(), torch.cuda.Stream()) if e2e else None

    def run(self, warmup, steps, clocks=None, skip=0):
        """skip: GP iterations run (untimed) before the warm-up, to time a
        later stage of the placement."""
        from dreamplace_b200._native import C
        warmup = warmup + skip
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        state = {"launch0": 0, "launch1": 0}
        pos = self.placer.pos[0]
        host_pos = torch.empty(pos.numel(), dtype=pos.dtype, pin_memory=True)

        def trials():
            st = getattr(self.placer, "stepper", None)
            eng = getattr(st, "eng", None)
            return eng.trials if eng is not None else 0

        def launches():
            st = getattr(self.placer, "stepper", None)
            eng = getattr(st, "eng", None)
            return eng.kernels_launched if eng is not None else C.launch_count()
        self.h2d = self.d2h = 0

        def cb(it, metric):
            if it == warmup - 1:
                eng = getattr(getattr(self.placer, "stepper", None), "eng", None)
                if eng is not None and eng.piece_events is not None:
                    # the warm-up trials timed every piece; the timed region
                    # accumulates only the longest one (one event query per trial)
                    means = eng.piece_means()
                    if means:
                        self.dominant = max(means, key=means.get)
                        # the timed trials carry the dominant piece's two events only
                        eng.time_only([self.dominant])
                torch.cuda.synchronize()
                barrier(self.world)
                torch.cuda.synchronize()
                if clocks is not None:
                    clocks.begin()
                state["launch0"] = launches()
                state["trials0"] = trials()
                start.record()
            elif warmup <= it < warmup + steps:
                if self.e2e:
                    # host round trip of the step's state: positions out and back in, metrics out
                    cur = self.placer.stepper.position()
                    host_round_trip(cur, host_pos, self.copy_streams)
                    self.h2d = host_pos.numel() * 4
                    self.d2h = host_pos.numel() * 4 + 3 * 8
                if it == warmup + steps - 1:
                    end.record()
                    torch.cuda.synchronize()
                    if clocks is not None:
                        clocks.end()
                    eng = getattr(getattr(self.placer, "stepper", None), "eng", None)
                    if self.dominant is not None and eng is not None:
                        self.dominant_ms = eng.piece_means().get(self.dominant)
                    state["launch1"] = launches()
                    state["trials1"] = trials()

        if clocks is not None:
            clocks.start()
        t0 = time.time()
        self.placer(self.params, self.design, max_iterations=warmup + steps, callback=cb)
        wall = time.time() - t0
        ms = start.elapsed_time(end)
        self.launches = state["launch1"] - state["launch0"]
        self.trials = state.get("trials1", 0) - state.get("trials0", 0)
        self.wall = wall
        return ms


E2E_CHUNKS = 8


def host_round_trip(dev, host, streams, chunks=E2E_CHUNKS):
    """dev -> pinned host -> dev, in order with the current stream: the
    download starts after the work already enqueued on it, and work enqueued
    after this call starts after the upload.  The buffer goes in `chunks`
    pieces on two copy streams, piece i's upload waiting only for piece i's
    download."""
    main = torch.cuda.current_stream()
    down, up = streams
    down.wait_stream(main)
    n = dev.numel()
    step = (n + chunks - 1) // chunks
    for a in range(0, n, step):
        b = min(a + step, n)
        with torch.cuda.stream(down):
            host[a:b].copy_(dev[a:b], non_blocking=True)
            done = torch.cuda.Event()
            done.record(down)
        up.wait_event(done)
        with torch.cuda.stream(up):
            dev[a:b].copy_(host[a:b], non_blocking=True)
    main.wait_stream(up)


def _graph_time(fn, reps=20):
    """Device time of fn per call: fn captured once in a CUDA graph, replayed reps times."""
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


def piece_work(design, eng):
    """Algorithmic bytes (or flops) of each piece of one Nesterov trial, per
    launch (n_s scattered cells, P pins, E nets, n nodes, M x N bins):

    * density_scatter: 28 B per scattered cell (16 B record + 4 B ratio + 8 B
      position); per bin 4 B initial map read and the two maps written (the
      movable-only map for the overflow and the movable + filler map);
    * poisson_gemms: the GEMM flops of one solve (three 2-D transforms, x3
      for split-BF16; the energy is summed in the spectral domain);
    * field_gather: per cell the same 28 B as the scatter + 8 B force written;
      per bin the two field maps read once;
    * wa_forward (HPWL included): per pin 12 B of pin arrays (node id, two
      offsets) + 8 B gradient written; per net 4 B start + 2 x 1 B masks +
      4 B weight; per node 8 B position (the pins' position gathers hit
      those 8 B);
    * assemble_precondition: per pin 8 B gradient read; per node 4 B pin
      start + 4 B inverse order + 8 B force + 4 B pin weight sum + 4 B area +
      3 x 8 B (v_new, v, g) read + 8 B written;
    * nesterov_trial: per node 3 x 8 B read (v, g, u) + 8 B cell size, 2 x 8 B
      written (u, v) + 8 B interleaved copy; per scattered cell 4 B order
      index + 8 B visiting-order copy written (the gather's re-read of the
      interleaved copy is not counted)."""
    from dreamplace_b200.electric_potential import poisson_flops
    d, ep = design, eng.ep
    n_s = d.num_movable_nodes + d.num_filler_nodes
    M, N = ep.num_bins_x, ep.num_bins_y
    P, E, n = d.num_pins, d.num_nets, d.num_nodes
    return {"density_scatter": (28.0 * n_s + 12.0 * M * N, "hbm"),
            "poisson_gemms": (poisson_flops(M, N, eng.prec), "tensor" if eng.prec else "fp32"),
            "field_gather": (36.0 * n_s + 8.0 * M * N, "hbm"),
            "wa_forward": (20.0 * P + 10.0 * E + 8.0 * n, "hbm"),
            "assemble_precondition": (8.0 * P + 64.0 * n, "hbm"),
            "nesterov_trial": (56.0 * n + 12.0 * n_s, "hbm")}


def kernel_roofline(placer, design, peaks, reps=20):
    """Device time of each piece of one Nesterov trial of the engine, each piece
    graph-captured alone and replayed (warm L2), with its algorithmic work
    (piece_work)."""
    from dreamplace_b200.electric_potential import poisson_solve
    eng = placer.stepper.eng
    ep = eng.ep
    work = piece_work(design, eng)
    p = eng.slot
    q = eng.next_slot(p)
    v, g = eng.V[p], eng.G[p]
    vn, gn = eng.V[q], eng.G[q]
    torch.cuda.synchronize()  # the iteration enqueued ahead writes the slot after q
    saved = eng.S[p].clone()
    t = {}
    t["density_scatter"] = _graph_time(lambda: eng.scatter_maps(v, eng.O[q]), reps)
    rho = eng.dmap.mul(1.0 / (ep.bin_size_x * ep.bin_size_y))
    t["poisson_gemms"] = _graph_time(lambda: poisson_solve(rho, ep.bin_size_x, ep.bin_size_y, eng.prec), reps)
    ex, ey, _ = poisson_solve(rho, ep.bin_size_x, ep.bin_size_y, eng.prec)
    t["field_gather"] = _graph_time(lambda: eng.field_force(v, ex, ey), reps)
    t["wa_forward"] = _graph_time(lambda: eng.wirelength(v, eng.H[q]), reps)
    t["assemble_precondition"] = _graph_time(lambda: eng.assemble(v, g, vn, gn), reps)
    t["nesterov_trial"] = _graph_time(lambda: eng.nesterov_trial_only(p), reps)
    eng.S[p].copy_(saved)
    return {k: (t[k],) + work[k] for k in t}


def dropin_ops(placer, design, peaks, precision, reps=10):
    """The reference-facing modules timed alone at the current GP position:
    ElectricPotential forward + backward (density map, Poisson solve, field
    gather) in fp32-atomic and deterministic (int64) scatter modes, and PinPos
    + WeightedAverageWirelength forward + backward.  CUDA events around reps
    eager calls after one warm call.  Algorithmic bytes: the electric potential
    reads 28 B per scattered cell twice (scatter, gather) and writes 8 B of
    force, plus the bin maps (4 B init read, two 4 B maps written, two 4 B
    field maps read); the Poisson GEMMs are counted as flops.  WA: pin_pos
    reads 8 B per node and 12 B per pin (node id, offsets) and writes 8 B per
    pin; WA reads 8 B and writes 8 B per pin gradient, plus 10 B per net;
    the backward sums 8 B per pin into 8 B per node."""
    import numpy as np
    from dreamplace_b200.electric_potential import ElectricPotential, poisson_flops
    from dreamplace_b200.placement_ops import PinPos
    from dreamplace_b200.weighted_average_wirelength import WeightedAverageWirelength
    from dreamplace_b200._native import precision_code
    d = design
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    pos0 = placer.stepper.position().detach().clone()
    m, n = d.num_movable_nodes, d.num_nodes
    n_s = m + d.num_filler_nodes
    M, N = d.num_bins_x, d.num_bins_y
    hbm = peaks.get("hbm_gbs", 6650.0)
    out = {}

    def time_fn(fn):
        fn()
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(reps):
            fn()
        e.record()
        torch.cuda.synchronize()
        return s.elapsed_time(e) / reps

    bcx = t(d.bin_centers(d.xl, d.xh, d.bin_size_x))
    bcy = t(d.bin_centers(d.yl, d.yh, d.bin_size_y))
    sorted_map = t(np.argsort(d.node_size_x[:m], kind="stable").astype(np.int32))
    ep_bytes = 2 * 28.0 * n_s + 8.0 * n_s + 4.0 * M * N * 5
    for det in (0, 1):
        ep = ElectricPotential(t(d.node_size_x), t(d.node_size_y), bcx, bcy, d.target_density, d.xl, d.yl, d.xh,
                               d.yh, d.bin_size_x, d.bin_size_y, m, d.num_terminals, d.num_filler_nodes, 0,
                               bool(det), sorted_map, precision=precision)
        pos = pos0.clone().requires_grad_(True)

        def ep_step():
            pos.grad = None
            ep(pos).backward()
        ms = time_fn(ep_step)
        out["electric_potential_" + ("deterministic" if det else "fp32_atomic")] = {
            "ms": round(ms, 4), "hbm_bytes": ep_bytes, "gemm_flop": poisson_flops(M, N, precision_code(precision)),
            "achieved_gbs_if_hbm_only": round(ep_bytes / (ms * 1e-3) / 1e9, 1)}
        del ep
    deg = np.diff(d.flat_net2pin_start_map)
    mask = ((deg >= 2) & (deg < 100)).astype(np.uint8)
    pin_pos = PinPos(t(d.pin_offset_x), t(d.pin_offset_y), t(d.pin2node_map), t(d.flat_node2pin_map),
                     t(d.flat_node2pin_start_map), d.num_physical_nodes)
    gamma = torch.tensor(4.0 * (d.bin_size_x + d.bin_size_y), device=dev)
    wa = WeightedAverageWirelength(t(d.flat_net2pin_map), t(d.flat_net2pin_start_map), t(d.pin2net_map),
                                   t(d.net_weights), t(mask), t(d.pin2node_map >= m), gamma, algorithm="merged")
    pos = pos0.clone().requires_grad_(True)

    def wa_step():
        pos.grad = None
        wa(pin_pos(pos)).backward()
    ms = time_fn(wa_step)
    P, E = d.num_pins, d.num_nets
    wa_bytes = 8.0 * n + 12.0 * P + 8.0 * P + 16.0 * P + 10.0 * E + 8.0 * P + 8.0 * n
    out["weighted_average_wirelength"] = {"ms": round(ms, 4), "hbm_bytes": wa_bytes,
                                          "achieved_gbs": round(wa_bytes / (ms * 1e-3) / 1e9, 1),
                                          "frac": round(wa_bytes / (ms * 1e-3) / 1e9 / hbm, 4)}
    out["timing"] = "CUDA events around %d eager forward + backward calls at the GP position of the timed run" % reps
    return out


def full_gp(design, precision, deterministic, max_iterations=3000):
    """Global placement of the design to the 0.07 overflow stop through the
    public placer; final metrics and wall time.  The 2.1M-cell design needs
    about 2,500 iterations to get there (its random 30% of far pins keep the
    HPWL-mode density-weight update slow), so the cap is 3,000."""
    from dreamplace_b200.nonlinear_place import place
    from dreamplace_b200.params import Params
    p = Params(target_density=design.target_density, stop_overflow=0.07, dct_precision=precision,
               deterministic_flag=int(deterministic))
    torch.cuda.synchronize()
    t0 = time.time()
    placer, res = place(design, p, device="cuda", max_iterations=max_iterations)
    torch.cuda.synchronize()
    res["wall_s"] = round(time.time() - t0, 3)
    res["iter_per_s_wall"] = round(res["iterations"] / res["wall_s"], 2)
    del placer
    return res


def full_gp_comparison(design, precision):
    """The metric's HPWL condition: the split-BF16 (or other) form and the
    plain fp32 form each run to the 0.07 overflow stop; their final HPWLs and
    the relative difference, in the benchmark's fp32-atomic scatter mode and
    in deterministic (int64 fixed-point) mode, where the two runs differ only
    in the Poisson-solve arithmetic."""
    out = {}
    for det in (0, 1):
        a = full_gp(design, precision, det)
        b = full_gp(design, "fp32", det)
        key = "deterministic" if det else "fp32_atomic"
        out[key] = {precision: a, "fp32": b,
                    "hpwl_rel_diff_final": round(abs(a["hpwl"] - b["hpwl"]) / b["hpwl"], 6)}
        torch.cuda.empty_cache()
    return out


def roofline_entry(name, ms, work, bound, peaks, timing):
    if bound == "hbm":
        achieved = work / (ms * 1e-3) / 1e9
        peak = peaks.get("hbm_gbs", 6650.0)
        unit = "GB/s"
    else:
        achieved = work / (ms * 1e-3) / 1e12
        peak = peaks.get("bf16_tflops", 1590.0) if bound == "tensor" else 74.0
        unit = "TFLOP/s"
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(name)
        except (OSError, ValueError):
            traffic = None
    return {"kernel": name, "bound": "hbm" if bound == "hbm" else "tensor", "achieved": round(achieved, 2),
            "peak": peak, "unit": unit, "frac": round(achieved / peak, 4), "traffic": traffic,
            "ms_per_launch": round(ms, 4), "work_per_launch": work, "timing": timing,
            "peak_source": "measured" if peaks else "fallback"}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return json.load(open(p))
    except (OSError, ValueError):
        return {}


# ------------------------------------------------------------------ reference CPU arm
class ReferenceCPUIteration(object):
    """One GP iteration composed from the reference's own CPU ops (oracle/_ref):
    HPWL + overflow evaluation, pin_pos, WA merged forward/backward, density map,
    the four dct2_fft2 transforms, electric force, preconditioning and the
    Nesterov vector update."""

    def __init__(self, design, threads):
        import oracle
        self.mods = {n: oracle.load_ref(n) for n in ("electric_potential_cpp", "dct2_fft2_cpp",
                                                     "weighted_average_wirelength_cpp_merged", "pin_pos_cpp",
                                                     "hpwl_cpp", "move_boundary_cpp", "pws_cpp")}
        missing = [k for k, v in self.mods.items() if v is None]
        if missing:
            raise RuntimeError("reference CPU ops not built: %s" % missing)
        torch.set_num_threads(threads)
        d = self.d = design
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a))  # noqa: E731
        self.pos = t(d.initial_positions())
        rng = np.random.RandomState(0)
        n, m = d.num_nodes, d.num_movable_nodes
        self.pos[:m] = torch.from_numpy(rng.uniform(d.xl, d.xh - 40, size=m).astype(np.float32))
        self.pos[n:n + m] = torch.from_numpy(rng.uniform(d.yl, d.yh - 12, size=m).astype(np.float32))
        self.sx, self.sy = t(d.node_size_x), t(d.node_size_y)
        bsx, bsy = d.bin_size_x, d.bin_size_y
        self.sxc = self.sx.clamp(min=bsx * math.sqrt(2))
        self.syc = self.sy.clamp(min=bsy * math.sqrt(2))
        self.ox = (self.sx - self.sxc).mul(0.5)
        self.oy = (self.sy - self.syc).mul(0.5)
        self.ratio = self.sx * self.sy / (self.sxc * self.syc)
        self.bcx = t(d.bin_centers(d.xl, d.xh, bsx))
        self.bcy = t(d.bin_centers(d.yl, d.yh, bsy))
        self.offx, self.offy = t(d.pin_offset_x), t(d.pin_offset_y)
        self.p2n = t(d.pin2node_map.astype(np.int64))
        self.fn2p, self.fn2ps = t(d.flat_node2pin_map), t(d.flat_node2pin_start_map)
        self.fnp, self.fnps = t(d.flat_net2pin_map), t(d.flat_net2pin_start_map)
        self.p2net = t(d.pin2net_map)
        self.w = t(d.net_weights)
        deg = np.diff(d.flat_net2pin_start_map)
        self.mask_all = t((deg >= 2).astype(np.uint8))
        self.mask = t(((deg >= 2) & (deg < 100)).astype(np.uint8))
        self.pin_mask = t(d.pin2node_map >= m)
        ep = self.mods["electric_potential_cpp"]
        self.init_map = ep.fixed_density_map(self.pos, self.sx, self.sy, self.bcx, self.bcy, d.xl, d.yl, d.xh, d.yh,
                                             bsx, bsy, m, d.num_terminals, d.num_bins_x, d.num_bins_y, 0, 0, 0)
        self.init_map.mul_(d.target_density)
        M, N = d.num_bins_x, d.num_bins_y
        u = torch.arange(M, dtype=torch.float32).mul_(np.pi / (2 * M))
        self.expkM = torch.stack([u.cos(), -u.sin()], -1).contiguous()
        v = torch.arange(N, dtype=torch.float32).mul_(np.pi / (2 * N))
        self.expkN = torch.stack([v.cos(), -v.sin()], -1).contiguous()
        wu = torch.arange(M, dtype=torch.float32).mul(2 * np.pi / M).view(M, 1)
        wv = torch.arange(N, dtype=torch.float32).mul(2 * np.pi / N).view(1, N).mul_(bsx / bsy)
        w2 = wu.pow(2) + wv.pow(2)
        w2[0, 0] = 1.0
        self.inv = 1.0 / w2
        self.inv[0, 0] = 0.0
        self.wx = wu.mul(self.inv).mul_(0.5)
        self.wy = wv.mul(self.inv).mul_(0.5)
        self.pws = self.mods["pws_cpp"].forward(self.w, self.fn2p, self.fn2ps, self.p2net, n)
        self.areas = self.sx * self.sy
        self.u_k = self.pos.clone()
        self.g_k = torch.zeros_like(self.pos)
        self.alpha = 1.0
        self.inv_gamma = torch.tensor([1.0 / (40 * (bsx + bsy))], dtype=torch.float32)

    def step(self):
        d, mo = self.d, self.mods
        ep, dct, wa, pp = mo["electric_potential_cpp"], mo["dct2_fft2_cpp"], mo[
            "weighted_average_wirelength_cpp_merged"], mo["pin_pos_cpp"]
        n, m, M, N = d.num_nodes, d.num_movable_nodes, d.num_bins_x, d.num_bins_y
        bsx, bsy = d.bin_size_x, d.bin_size_y
        threads = torch.get_num_threads()
        pos = self.pos
        mo["move_boundary_cpp"].forward(pos, self.sx, self.sy, d.xl, d.yl, d.xh, d.yh, m, d.num_filler_nodes)
        # evaluation
        pin = pp.forward(pos, self.offx, self.offy, self.p2n, self.fn2p, self.fn2ps)
        hp = mo["hpwl_cpp"].forward(pin, self.fnp, self.fnps, self.w, self.mask_all)
        dmo = ep.density_map(pos, self.sxc, self.syc, self.ox, self.oy, self.ratio, self.bcx, self.bcy,
                             self.init_map, d.target_density, d.xl, d.yl, d.xh, d.yh, bsx, bsy, m, 0, 0, M, N,
                             0, 0, 0, 0, 0)
        ovf = (dmo - d.target_density * bsx * bsy).clamp_(min=0).sum()
        # objective and gradient
        pin = pp.forward(pos, self.offx, self.offy, self.p2n, self.fn2p, self.fn2ps)
        wl, gi = wa.forward(pin, self.fnp, self.fnps, self.p2net, self.w, self.mask, self.inv_gamma)
        dm = ep.density_map(pos, self.sxc, self.syc, self.ox, self.oy, self.ratio, self.bcx, self.bcy,
                            self.init_map, d.target_density, d.xl, d.yl, d.xh, d.yh, bsx, bsy, m,
                            d.num_filler_nodes, 0, M, N, 0, 0, 0, 0, 0)
        rho = dm.view(M, N).mul_(1.0 / (bsx * bsy))
        buf = torch.empty(M, N // 2 + 1, 2)
        auv, ex, ey, phi = (torch.empty(M, N) for _ in range(4))
        dct.dct2_fft2(rho, self.expkM, self.expkN, auv, buf, threads)
        dct.idxst_idct(auv.mul(self.wx), self.expkM, self.expkN, ex, buf, threads)
        dct.idct_idxst(auv.mul(self.wy), self.expkM, self.expkN, ey, buf, threads)
        dct.idct2_fft2(auv.mul(self.inv), self.expkM, self.expkN, phi, buf, threads)
        energy = phi.mul(rho).sum()
        one = torch.ones(1)
        gd = -ep.electric_force(one, M, N, 0, 0, 0, 0, ex.view(-1), ey.view(-1), pos, self.sxc, self.syc, self.ox,
                                self.oy, self.ratio, self.bcx, self.bcy, d.xl, d.yl, d.xh, d.yh, bsx, bsy, m,
                                d.num_filler_nodes)
        gw = wa.backward(one, pin, gi, self.fnp, self.fnps, self.p2net, self.w, self.mask, self.inv_gamma)
        gw[:d.num_pins].masked_fill_(self.pin_mask, 0.0)
        gw[d.num_pins:].masked_fill_(self.pin_mask, 0.0)
        gpos = pp.backward(gw, pos, self.offx, self.offy, self.p2n, self.fn2p, self.fn2ps, d.num_physical_nodes)
        grad = gpos + 1e-3 * gd
        precond = (self.pws + 1e-3 * self.areas).clamp_(min=1.0)
        grad.view(2, n).div_(precond)
        # Nesterov vector update and step-size estimate
        u = pos - self.alpha * grad
        v = u + 0.5 * (u - self.u_k)
        a = torch.sqrt(torch.sum((v - pos) ** 2) / torch.sum((grad - self.g_k) ** 2).clamp_(min=1e-30))
        self.u_k.copy_(u)
        self.g_k.copy_(grad)
        pos.copy_(pos + 1e-6 * (v - pos))
        return float(hp) + float(ovf) + float(wl) + float(energy) + float(a)


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def time_reference_cpu(design, steps, threads):
    it = ReferenceCPUIteration(design, threads)
    it.step()  # warm-up
    t0 = time.time()
    for _ in range(steps):
        it.step()
    return steps / (time.time() - t0)


def run_reference(args):
    rank, local, world = int(os.environ.get("RANK", "0")), 0, int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    design = make_design(args.design)
    threads = cpu_threads()
    it = ReferenceCPUIteration(design, threads)
    for _ in range(max(args.warmup, 1)):
        it.step()
    steps = args.steps
    t0 = time.time()
    for _ in range(steps):
        it.step()
    dt = time.time() - t0
    value = steps / dt
    line = {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": round(1000 * dt / steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": design.name + ": %d movable cells, %d nets, %d pins, %dx%d bins"
                       % (design.num_movable_nodes, design.num_nets, design.num_pins, design.num_bins_x,
                          design.num_bins_y), "parallelism": "host threads"},
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": "%d GP iterations composed from the reference CPU ops (%s)"
                                       % (steps, cpu_model())},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ main
def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    rank, local, world = dist_setup(args.gpus)
    design = make_design(args.design)
    peaks = load_peaks()
    W, K = max(args.warmup, 3), args.steps
    clocks = ClockSampler(local) if rank == 0 else None
    spec = not args.no_speculate
    if args.process_warmup > 0:
        # an untimed GP run of the same design first: the timed run then starts
        # with the process's one-time costs (lazy kernel loading, allocator
        # growth, first-call host paths) behind it, as every later run does
        pre = TimedRun(design, args.precision, world, speculate=spec)
        pre.run(3, args.process_warmup)
        del pre
        torch.cuda.empty_cache()
    run = TimedRun(design, args.precision, world, time_pieces=not args.no_roofline, speculate=spec)
    ms = run.run(W, K, clocks=clocks, skip=args.skip_to)
    clk = clocks.stop() if clocks else None
    ms = max_over_ranks(ms, world)
    value = replica_value(K, world, ms)
    launches = run.launches
    # end-to-end through the public API with a host round trip per step
    e2e = None
    if not args.no_e2e:
        run_e2e = TimedRun(design, args.precision, world, e2e=True, speculate=spec)
        ms_e2e = max_over_ranks(run_e2e.run(W, K), world)
        e2e = {"value": round(replica_value(K, world, ms_e2e), 3), "unit": UNIT,
               "h2d_bytes_per_step": run_e2e.h2d, "d2h_bytes_per_step": run_e2e.d2h}
    pieces = {} if args.no_roofline else kernel_roofline(run.placer, design, peaks)
    dropin = None if args.no_dropin else dropin_ops(run.placer, design, peaks, args.precision)
    roof = None
    if run.dominant is not None and run.dominant_ms:
        work, bound = piece_work(design, run.placer.stepper.eng)[run.dominant]
        roof = roofline_entry(run.dominant, run.dominant_ms, work, bound, peaks,
                              "CUDA events around the piece inside the captured trial graph, mean over the "
                              "trials of the timed region")
    plain = None
    if not args.no_plain and args.precision != "fp32":
        prun = TimedRun(design, "fp32", world, speculate=spec)
        pms = max_over_ranks(prun.run(W, K), world)
        pval = world * K / (pms / 1000.0)
        h_ours = run.placer.metrics[-1][-1][-1]._host[0]
        h_plain = prun.placer.metrics[-1][-1][-1]._host[0]
        plain = {"value": round(pval, 3), "ms_per_step": round(pms / K, 3), "speedup": round(value / pval, 3),
                 "hpwl_rel_diff_at_step": round(abs(h_ours - h_plain) / h_plain, 6), "compared_at_iteration": W + K}
    kernels = {}
    if pieces:
        for k, (kms, work, bound) in pieces.items():
            e = roofline_entry(k, kms, work, bound, peaks, "piece captured alone, replayed 20x")
            kernels[k] = {"ms": e["ms_per_launch"], "achieved": e["achieved"], "unit": e["unit"], "frac": e["frac"],
                          "bound": e["bound"], "work_per_launch": work}
    convergence = None
    if not args.no_full_gp and args.precision != "fp32":
        run.placer = None  # free the timed runs' design state first
        run_e2e = prun = None  # noqa: F841
        torch.cuda.empty_cache()
        convergence = full_gp_comparison(design, args.precision)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        threads = cpu_threads()
        try:
            v = time_reference_cpu(design, args.cpu_sample_steps, threads)
            cpu = {"value": round(v, 4), "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": "%d GP iterations composed from the reference CPU ops at the same design (%s)"
                             % (args.cpu_sample_steps, cpu_model())}
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": threads, "kind": "reference", "sample": "failed: %s" % e}
    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
                "ms_per_step": round(ms / K, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32+" + args.precision, "data": "synthetic",
                "config": {"workload": "%s: %d movable cells, %d macros, %d fillers, %d nets, %d pins, %dx%d bins"
                           % (design.name, design.num_movable_nodes, design.num_terminals, design.num_filler_nodes,
                              design.num_nets, design.num_pins, design.num_bins_x, design.num_bins_y),
                           "dct_precision": args.precision, "parallelism": "replicas%d" % world,
                           "l2": "per-iteration working set > 126 MB L2, no flush",
                           "process_warmup": "%d untimed GP iterations of the same design in a separate run "
                                             "before the timed run" % args.process_warmup},
                "e2e": e2e,
                "gpu_launches": int(launches), "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
                "kernel_ms": {k: round(v[0], 4) for k, v in pieces.items()},
                "kernel_ms_timing": "each piece captured alone and replayed 20x after the timed region",
                "kernels": kernels,
                "trials_per_step": round(run.trials / max(K, 1), 3),
                "voided_speculative_trials": int(run.trials - K),
                "plain_fp32": plain,
                "dropin_ops": dropin,
                "full_gp_to_overflow_0.07": convergence,
                "hpwl_rel_diff_final": (convergence["fp32_atomic"]["hpwl_rel_diff_final"]
                                        if convergence else None)}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
