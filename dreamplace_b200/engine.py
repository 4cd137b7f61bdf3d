"""Graph-captured global-placement iteration.

The same iteration as ``NonLinearPlace`` + ``NesterovAcceleratedGradientOptimizer``
(dreamplace/NonLinearPlace.py:377-526, dreamplace/NesterovAcceleratedGradientOptimizer.py:65-166),
re-organised for the GPU:

* the objective and its gradient are computed by the hand-written adjoints
  directly (no autograd): WA forward with the pin gather fused in, the density
  scatter, the four Poisson GEMM launches, the field gather writing the
  density gradient (scaled by lambda on the device) and the WA backward fused
  with the pin -> node sum accumulating the wirelength gradient on top;
* the Nesterov trial point, move-boundary clamp, preconditioner and the fp64
  step-size estimate run as fused kernels on three rotating slots of (v, u, g)
  buffers, so an accepted step advances a slot index instead of copying;
* one Nesterov trial is one CUDA graph replay; the trial's WA forward also
  sums the HPWL of the trial point and its scatter also yields the
  movable-only map, so the evaluation of v_k (HPWL, overflow) reported at
  iteration k was computed when v_k was produced; the host reads a handful of
  fp64 scalars once per trial and makes the loop decisions;
* the loop's between-iteration work (Nesterov advance, density-weight and
  gamma updates) runs on the device at the head of the next iteration's graph,
  so iteration k+1 is enqueued before the host has read iteration k: the host
  loop runs while the GPU computes, and iteration k+1 is enqueued again only
  when k needed a retry or the host changed what k+1 reads.
"""
import math

import numpy as np
import torch

from ._native import C, precision_code
from .electric_potential import PoissonWorkspace, poisson_solve

# device scalar slots of the optimizer state (gp_step.cu)
NS_ALPHA, NS_A, NS_A_NEXT, NS_COEF, NS_ACC_DV, NS_ACC_DG, NS_ALPHA_NEW, NS_ACCEPT = range(8)
NESTEROV_STATE = 8
REDUCE_DOUBLES = 1280
NSLOT = 3
# metric slots
M_HPWL, M_OVF, M_MAXD, M_ACCEPT, M_ALPHA, M_OBJ, M_WL, M_ENERGY = range(8)
# pieces of one Nesterov trial, in launch order
PIECES = ("nesterov_trial", "wa_forward", "density_scatter", "poisson_gemms", "field_gather", "assemble_precondition")


class GPEngine(object):
    def __init__(self, params, design, data, ops, model, use_graphs=True):
        self.params = params
        self.design = d = design
        self.data = data
        self.ops = ops
        self.model = model
        self.use_graphs = use_graphs
        dev = data.pos[0].device
        self.dev = dev
        self._dev_index = dev.index if dev.index is not None else torch.cuda.current_device()
        self._stream_raw = None
        self._stream_obj = None
        n = d.num_nodes
        P = d.num_pins
        fnp = data.flat_net2pin_map.long()
        self.slot_node = data.pin2node_map[fnp].to(torch.int32).contiguous()
        self.slot_offx = data.pin_offset_x[fnp].contiguous()
        self.slot_offy = data.pin_offset_y[fnp].contiguous()
        slot_of_pin = torch.empty(P, dtype=torch.int64, device=dev)
        slot_of_pin[fnp] = torch.arange(P, device=dev)
        self.node_slots = slot_of_pin[data.flat_node2pin_map.long()].to(torch.int32).contiguous()
        self.node_start = data.flat_node2pin_start_map
        self.netpin_start = data.flat_net2pin_start_map
        # each pin's position in node-CSR order (where the assembly reads its gradient)
        csr_pos = torch.empty(P, dtype=torch.int64, device=dev)
        csr_pos[self.node_slots.long()] = torch.arange(P, device=dev)
        self.csr_pos = csr_pos.to(torch.int32)
        self.gnode = torch.empty(2 * P, dtype=torch.float32, device=dev)
        # lane-per-net plan: nets of degree <= 8 grouped 32 at a time by degree,
        # pin arrays gathered into the transposed lane-slot order
        self.net_order = getattr(params, "net_order", "locality")
        order = self._net_locality_order() if self.net_order == "locality" else None
        g_deg, g_base, g_net, l_slot = C.plan_net_lanes(self.netpin_start.cpu(), order)
        self.group_deg, self.group_base, self.group_net = g_deg.to(dev), g_base.to(dev), g_net.to(dev)
        ls = l_slot.to(dev).long()
        real = ls >= 0
        ls = ls.clamp(min=0)
        self.ln_node = torch.where(real, self.slot_node[ls], torch.zeros_like(self.slot_node[ls])).contiguous()
        self.ln_offx = torch.where(real, self.slot_offx[ls], torch.zeros_like(self.slot_offx[ls])).contiguous()
        self.ln_offy = torch.where(real, self.slot_offy[ls], torch.zeros_like(self.slot_offy[ls])).contiguous()
        self.ln_csr = torch.where(real, self.csr_pos[ls], torch.zeros_like(self.csr_pos[ls])).contiguous()
        # where the WA gradient lands: "csr" (node-CSR order, scattered writes)
        # or "lane" (lane-slot order, coalesced writes; the assembly gathers it)
        self.wa_grad_order = getattr(params, "wa_grad_order", "lane")
        self.lane_of_csr = None
        if self.wa_grad_order == "lane":
            p_idx = torch.arange(ls.numel(), device=dev)[real]
            self.lane_of_csr = torch.empty(P, dtype=torch.int32, device=dev)
            self.lane_of_csr[self.csr_pos[ls[real]].long()] = p_idx.to(torch.int32)
            self.gnode = torch.empty(2 * ls.numel(), dtype=torch.float32, device=dev)
        ep = ops.density_op
        self.ep = ep
        self.ovf_op = ops.density_overflow_op
        # iteration slots: slot s holds v_k, u_k, g_k of an iteration (and its
        # interleaved / visiting-order position copies, the HPWL and overflow
        # of v_k, the optimizer scalars, the density weight and gamma); a trial
        # reads slot s and writes slot s + 1 (mod 3).  Three slots let
        # iteration k+1 be enqueued while iteration k may still be retried.
        pos = data.pos[0]
        self.V = [pos.data.clone()] + [torch.empty_like(pos.data) for _ in range(NSLOT - 1)]
        self.U = [torch.empty_like(pos.data) for _ in range(NSLOT)]
        self.G = [torch.empty_like(pos.data) for _ in range(NSLOT)]
        # interleaved (x, y) copies of the positions for the gather kernels
        self.XY = [torch.empty_like(pos.data) for _ in range(NSLOT)]
        self._xy_of = {self.V[i].data_ptr(): self.XY[i] for i in range(NSLOT)}
        # the same positions for the scattered cells, in visiting order (written
        # by the trial kernel; gathered after a pack or a re-sort)
        ns = d.num_movable_nodes + d.num_filler_nodes
        self.XYO = [torch.empty(2 * ns, dtype=torch.float32, device=dev) for _ in range(NSLOT)]
        self._xyo_of = {self.V[i].data_ptr(): self.XYO[i] for i in range(NSLOT)}
        self.tmp = torch.empty_like(pos.data)
        f64 = dict(dtype=torch.float64, device=dev)
        # optimizer scalars + fixed-order reduction scratch (include/dreamplace_b200.h)
        self.S = [torch.zeros(NESTEROV_STATE + 2 * REDUCE_DOUBLES, **f64) for _ in range(NSLOT)]
        # {iteration index, HPWL of the previous iteration} and {lambda, gamma,
        # 1 / gamma} of the iteration in each slot (dp_iteration_head)
        self.sched = [torch.zeros(2, **f64) for _ in range(NSLOT)]
        self.weights = [torch.zeros(3, dtype=torch.float32, device=dev) for _ in range(NSLOT)]
        self.wl64_buf = torch.zeros(REDUCE_DOUBLES, **f64)
        self.wl64 = self.wl64_buf[0:1]
        self.obj64 = torch.zeros(1, **f64)
        # metrics of v_k by slot: the HPWL rides along the WA forward of the trial
        # that produced v_k and the movable-only map (overflow) along its
        # scatter, so the evaluation of v_k is on the device when iteration k starts
        self.H = [torch.zeros(REDUCE_DOUBLES, **f64) for _ in range(NSLOT)]
        self.O = [torch.zeros(REDUCE_DOUBLES, **f64) for _ in range(NSLOT)]
        self.metrics = [torch.zeros(8, **f64) for _ in range(NSLOT)]
        self.metrics_host = [torch.zeros(8, dtype=torch.float64, pin_memory=True) for _ in range(NSLOT)]
        self.ready = [None] * NSLOT
        self.grad_scale = torch.zeros(1, dtype=torch.float32, device=dev)
        # (density factor, quadratic penalty coefficient) read by the objective
        # kernel on the device, so the captured graphs follow their changes
        self.factor_quad = torch.tensor([1.0, 0.0], dtype=torch.float32, device=dev)
        self.one = torch.ones(1, dtype=torch.float32, device=dev)
        self.inv_gamma = torch.zeros(1, dtype=torch.float32, device=dev)  # set-up evaluations (model gamma)
        self.dmap = torch.empty(ep.num_bins_x, ep.num_bins_y, dtype=torch.float32, device=dev)
        self.omap = torch.empty_like(self.dmap)
        self.ovf_area = float(self.ovf_op.bin_size_x * self.ovf_op.bin_size_y)
        self.ovf_target = float(self.ovf_op.target_density) * self.ovf_area
        self.det = bool(params.deterministic_flag)
        self.scratch = torch.empty(ep.num_bins_x * ep.num_bins_y, dtype=torch.int64, device=dev) if self.det else None
        self.prec = precision_code(ep.precision)
        # the Poisson solve's operands and outputs, allocated once: every trial
        # (eager or captured) of this design solves on its one stream
        self.poisson_ws = PoissonWorkspace(ep.num_bins_x, ep.num_bins_y, self.prec, dev)
        # spatial visiting order of the scattered cells (movable block, then filler
        # block), refreshed every `sort_interval` iterations (refresh_due)
        nm, nf = d.num_movable_nodes, d.num_filler_nodes
        self.order = torch.cat([torch.arange(nm, device=dev), torch.arange(n - nf, n, device=dev)]).to(torch.int32)
        # per-cell records in that order (stretched size, offset, ratio), the
        # inverse order, and the field force in order space
        count = nm + nf
        self.rec4 = torch.empty(4 * count, dtype=torch.float32, device=dev)
        self.ratio_o = torch.empty(count, dtype=torch.float32, device=dev)
        self.inv_order = torch.zeros(n, dtype=torch.int32, device=dev)
        self.force_o = torch.empty(2 * count, dtype=torch.float32, device=dev)
        nbytes = C.order_cells_scratch_bytes(nm, nf, ep.num_bins_x, ep.num_bins_y)
        self.order_scratch = torch.empty((nbytes + 3) // 4, dtype=torch.int32, device=dev)
        self._build_records()
        # every 25 iterations (2.1M-cell design, 1024^2 bins: 1848 GP iter/s over
        # iterations 5..305 against 1710 at every 50 and 1788 at every 10 up to
        # iteration 200); sort_schedule: optional (until_iteration, interval)
        # pairs applied before sort_interval
        self.sort_interval = int(getattr(params, "sort_interval", 25))
        self.sort_schedule = [tuple(int(v) for v in x) for x in getattr(params, "sort_schedule", ())]
        # how the scatter and the field gather read the trial point: "gather"
        # (a visiting-order copy gathered after the trial), "trial" (the copy
        # written by scattered stores in the trial kernel) or "order" (no copy:
        # the kernels read the node-order positions through the order)
        self.xyo_mode = getattr(params, "xyo_mode", "gather")
        if self.xyo_mode not in ("gather", "trial", "order"):
            raise ValueError("xyo_mode must be 'gather', 'trial' or 'order'")
        # optional per-piece device timing of the trial (CUDA events recorded
        # inside the captured graph); piece_query selects the pieces whose
        # durations are accumulated after each trial
        self.piece_events = None
        self._mark_slot = 0
        self.piece_query = set(PIECES)
        self.piece_record = set(PIECES)  # pieces whose events the captured trials record
        self.piece_ms = {k: 0.0 for k in PIECES}
        self.piece_n = {k: 0 for k in PIECES}
        if getattr(params, "time_pieces", False):
            # one set per slot: the trial of the next slot may record its own
            # while this slot's durations are read
            self.piece_events = [{k: (torch.cuda.Event(enable_timing=True, external=True),
                                      torch.cuda.Event(enable_timing=True, external=True)) for k in PIECES}
                                 for _ in range(NSLOT)]
        self.iterations = 0
        self.slot = 0
        # the iteration whose first trial is already enqueued (None: none)
        self.enqueued = None
        # enqueue iteration k+1 right behind iteration k's first trial, before the
        # host has read k's metrics (the GP loop's between-iteration work runs on
        # the device, dp_iteration_head); needs the loop's default schedule of one
        # Nesterov step per density-weight and per gamma update
        gp = params.global_place_stages[0]
        self.schedule_ok = int(gp.get("Lsub_iteration", 1)) == 1 and \
            int(gp.get("Llambda_density_weight_iteration", 1)) == 1
        if not self.schedule_ok:
            raise ValueError("the graph engine runs the default schedule (Lsub_iteration = "
                             "Llambda_density_weight_iteration = 1); use gp_engine='autograd' for others")
        self.speculate = bool(getattr(params, "speculate", True)) and use_graphs
        # trial gate word (dp_set_trial_gate): written by each trial graph's
        # first kernel; a trial enqueued ahead of a rejected one skips its work
        self.gate = torch.zeros(1, dtype=torch.int32, device=dev)
        self.head_scalars = (float(model.base_gamma(params, d)), float(d.total_movable_node_area),
                             float(params.RePlAce_ref_hpwl), float(params.RePlAce_LOWER_PCOF),
                             float(params.RePlAce_UPPER_PCOF))
        self.graphs = {}
        self.graph_exec = {}  # raw cudaGraphExec_t of each captured trial
        self.graph_kernels = {}
        self.kernels_launched = 0  # this library's kernels, graph replays included
        # best position so far (the GP loop's divergence rollback target): the
        # slot that holds it and the buffer it is copied into before that slot
        # is overwritten; a newer best usually supersedes it first, so most
        # improvements cost no copy
        self.best_slot = None
        self.best_buf = None
        self.pool = None
        self.graph_key = None
        self.trials = 0
        self.last_energy = None
        self._quad_c = 0.0

    def _net_locality_order(self):
        """Nets ordered by the median node index of their pins (CPU int32
        permutation for the lane planner).  Nets whose pins sit on nearby nodes
        then share lane groups and neighbouring lane slots, so the WA kernel's
        position gathers and the assembly's gradient gather stay local; the
        median ignores a net's few far-away pins."""
        ns = self.netpin_start.long()
        num_nets = ns.numel() - 1
        deg = ns[1:] - ns[:-1]
        if num_nets == 0 or int(ns[-1]) == 0:
            return None
        span = int(self.design.num_nodes) + 1
        net_of_slot = torch.repeat_interleave(torch.arange(num_nets, device=ns.device), deg)
        key = torch.sort(net_of_slot * span + self.slot_node.long()).values
        mid = (ns[:-1] + deg // 2).clamp(max=key.numel() - 1)
        median = key[mid] - torch.arange(num_nets, device=ns.device) * span
        median = torch.where(deg > 0, median, torch.zeros_like(median))
        return torch.argsort(median, stable=True).to(torch.int32).cpu()

    # ---------------------------------------------------------------- pieces
    def _build_records(self):
        ep = self.ep
        C.build_cell_records(ep.node_size_x_clamped, ep.node_size_y_clamped, ep.offset_x, ep.offset_y, ep.ratio,
                             self.order, self.order.numel(), self.rec4, self.ratio_o, self.inv_order)

    def _density(self, v, num_filler, out):
        ep = self.ep
        count = ep.num_movable_nodes + (num_filler if num_filler else 0)
        xy_o, order = self._cells_xy(v)
        C.density_map_ordered_into(xy_o, self.rec4, self.ratio_o, count,
                                   ep.initial_density_map.view(-1), float(ep.xl), float(ep.yl), float(ep.xh),
                                   float(ep.yh), float(ep.bin_size_x), float(ep.bin_size_y), ep.num_bins_x,
                                   ep.num_bins_y, int(self.det), self.scratch, out, order=order)

    def refresh_order(self, v):
        """Sort movable and filler cells by the bin where their stretched footprint
        starts: 16x16-bin tiles in serpentine order (neighbouring tiles follow each
        other), then bin inside the tile.  Each scatter block's cells then cover a
        compact patch of bins, and cells with the same start bin are adjacent."""
        d, ep = self.design, self.ep
        nm, nf = d.num_movable_nodes, d.num_filler_nodes
        with torch.no_grad():
            # counting sort by start bin (dp_order_cells_by_bin)
            C.order_cells_by_bin(v, ep.offset_x, ep.offset_y, nm, nf, float(ep.xl), float(ep.yl),
                                 float(ep.bin_size_x), float(ep.bin_size_y), ep.num_bins_x, ep.num_bins_y,
                                 self.order_scratch, self.order)
            self._build_records()
            if self.xyo_mode != "order":
                C.gather_order_xy(self.xy(v), self.order, self.order.numel(), self.xyo(v))

    def xy(self, v):
        return self._xy_of[v.data_ptr()]

    def xyo(self, v):
        return self._xyo_of[v.data_ptr()]

    def _cells_xy(self, v):
        """(positions, order) for the scatter and the field gather: the
        visiting-order copy, or (xyo_mode "order") the node-order interleaved
        copy read through the visiting order."""
        if self.xyo_mode == "order":
            return self.xy(v), self.order
        return self.xyo(v), None

    def pack(self, v):
        """Refresh the interleaved and the visiting-order copies of a position buffer
        written outside the trial kernel."""
        C.pack_xy(v, self.xy(v))
        if self.xyo_mode != "order":
            C.gather_order_xy(self.xy(v), self.order, self.order.numel(), self.xyo(v))

    def wirelength(self, v, hpwl_out=None, inv_gamma=None):
        """WA forward at node positions v: fp64 total in self.wl64, per-pin gradient (times the
        net weight) in self.gnode; with hpwl_out, the HPWL of v from the same pin reads.
        inv_gamma: device scalar 1/gamma (default: from the model's gamma)."""
        dc = self.data
        if inv_gamma is None:
            self.inv_gamma.copy_(1.0 / self.model.gamma.reshape(1))
            inv_gamma = self.inv_gamma
        C.wa_lanes_forward(self.xy(v), self.group_deg, self.group_base, self.group_net, self.ln_node, self.ln_offx,
                           self.ln_offy, self.ln_csr if self.lane_of_csr is None else None, dc.net_weights,
                           dc.net_mask_ignore_large_degrees,
                           inv_gamma, self.wl64_buf, self.gnode,
                           dc.net_mask_all if hpwl_out is not None else None, hpwl_out)

    def wl_grad_into(self, g, accumulate):
        gn = self.gnode
        if self.lane_of_csr is not None:  # lane-slot order -> node-CSR order
            gn = gn.view(-1, 2)[self.lane_of_csr.long()].reshape(-1).contiguous()
        C.node_pin_sum(gn, self.node_start, self.one, self.design.num_movable_nodes, int(accumulate), g)

    def scatter_maps(self, v, ovf_out):
        """One scatter of v: the movable-only map (self.omap) and the movable +
        filler map (self.dmap); (overflow, max density) of v into ovf_out."""
        ep = self.ep
        xy_o, order = self._cells_xy(v)
        C.density_map_ordered_split(xy_o, self.rec4, self.ratio_o, ep.num_movable_nodes,
                                    self.order.numel(), ep.initial_density_map.view(-1), float(ep.xl), float(ep.yl),
                                    float(ep.xh), float(ep.yh), float(ep.bin_size_x), float(ep.bin_size_y),
                                    ep.num_bins_x, ep.num_bins_y, int(self.det), self.scratch, self.omap.view(-1),
                                    self.dmap.view(-1), self.ovf_target, self.ovf_area, ovf_out, order=order)

    def density_energy(self, v, ovf_out=None):
        """Density map, Poisson solve; returns (ex, ey, energy_f64[1]).  With ovf_out,
        the movable-only map of the same scatter gives (overflow, max density) of v."""
        ep = self.ep
        if ovf_out is None:
            self._density(v, ep.num_filler_nodes, self.dmap)
        else:
            self.scatter_maps(v, ovf_out)
        self.dmap.mul_(1.0 / (ep.bin_size_x * ep.bin_size_y))
        return poisson_solve(self.dmap, ep.bin_size_x, ep.bin_size_y, self.prec, bool(ep.fast_mode),
                             ws=self.poisson_ws)

    def field_force(self, v, ex, ey):
        """Field force of every movable and filler cell, in visiting order (self.force_o)."""
        ep = self.ep
        xy_o, order = self._cells_xy(v)
        C.electric_force_ordered(self.grad_scale, ex.view(-1), ey.view(-1), xy_o, self.rec4,
                                 self.ratio_o, self.order.numel(), float(ep.xl), float(ep.yl), float(ep.bin_size_x),
                                 float(ep.bin_size_y), ep.num_bins_x, ep.num_bins_y, -1.0, self.force_o, order=order)

    def assemble(self, v, g, v_new, g_new, s=None):
        """Preconditioned gradient at v_new into g_new (pin sum + force) and the fp64
        step-size norms against (v, g), with the density weight and optimizer
        scalars of slot s (default: the current slot)."""
        d = self.design
        s = self.slot if s is None else s
        C.assemble_precondition_step(self.gnode, self.node_start, self.one, self.force_o, self.inv_order,
                                     d.num_movable_nodes, d.num_filler_nodes, self._pws(), self.data.node_areas,
                                     self.weights[s][0:1], v_new, v, g, g_new, self.S[s], self.lane_of_csr)

    def density_grad_into(self, v, ex, ey, scale_t, g):
        ep = self.ep
        C.electric_force_into(scale_t, ex.view(-1), ey.view(-1), v, ep.node_size_x_clamped, ep.node_size_y_clamped,
                              ep.offset_x, ep.offset_y, ep.ratio, float(ep.xl), float(ep.yl), float(ep.xh),
                              float(ep.yh), float(ep.bin_size_x), float(ep.bin_size_y), ep.num_bins_x, ep.num_bins_y,
                              ep.num_movable_nodes, ep.num_filler_nodes, ep.sorted_node_map, -1.0, g)

    def obj_and_raw_grad(self, v, g):
        """obj (fp64, self.obj64) and the un-preconditioned gradient into g."""
        m = self.model
        self.wirelength(v)
        ex, ey, energy = self.density_energy(v)
        C.objective_finish(self.wl64, energy, m.density_weight, self.factor_quad, self.obj64, self.grad_scale)
        self.density_grad_into(v, ex, ey, self.grad_scale, g)
        self.wl_grad_into(g, True)
        self.last_energy = energy
        return energy

    def _pws(self):
        m = self.model
        if m.ops.precondition_op._pws is None:
            m.ops.precondition_op._pws = m.ops.pws_op(self.data.net_weights)
        return m.ops.precondition_op._pws

    def precondition(self, g, v_ref, g_ref, v_new):
        C.precondition_step_size(g, g_ref, v_new, v_ref, self._pws(), self.data.node_areas,
                                 self.model.density_weight, self.S[self.slot])

    def objective_and_step(self, v, g, v_new, g_new, s):
        """The trial's objective at v_new and its preconditioned gradient into g_new,
        with the fp64 step-size norms against (v, g) into slot s's scalars: the
        field force is gathered in visiting order and assembled per node together
        with the wirelength pin sum, the preconditioner and the norms (one pass
        over the nodes).  The HPWL and overflow of v_new land in the metric
        buffers of slot s + 1."""
        ep = self.ep
        q_new = (s + 1) % NSLOT
        w = self.weights[s]
        # (the WA forward was also run on a second stream beside the density
        # chain: its kernels and the scatter's, or the GEMMs', slow each other
        # down by about what they would overlap, ~1% net, so it runs in line)
        self._mark("wa_forward", 0)
        self.wirelength(v_new, self.H[q_new], w[2:3])
        self._mark("wa_forward", 1)
        self._mark("density_scatter", 0)
        self.scatter_maps(v_new, self.O[q_new])
        self._mark("density_scatter", 1)
        self._mark("poisson_gemms", 0)
        # rho = D / bin area is applied as the first GEMM's alpha
        ex, ey, energy = poisson_solve(self.dmap, ep.bin_size_x, ep.bin_size_y, self.prec, bool(ep.fast_mode),
                                       1.0 / (ep.bin_size_x * ep.bin_size_y), self.poisson_ws)
        self._mark("poisson_gemms", 1)
        C.objective_finish(self.wl64, energy, w[0:1], self.factor_quad, self.obj64, self.grad_scale)
        self._mark("field_gather", 0)
        self.field_force(v_new, ex, ey)
        self._mark("field_gather", 1)
        self._mark("assemble_precondition", 0)
        self.assemble(v, g, v_new, g_new, s)
        self._mark("assemble_precondition", 1)
        self.last_energy = energy
        return energy

    def _mark(self, piece, which):
        if self.piece_events is not None and piece in self.piece_record:
            self.piece_events[self._mark_slot][piece][which].record()

    def _collect_pieces(self, s):
        for k in self.piece_query:
            a, b = self.piece_events[s][k]
            self.piece_ms[k] += a.elapsed_time(b)
            self.piece_n[k] += 1

    def reset_piece_times(self, query=None):
        self.piece_query = set(PIECES) if query is None else set(query)
        self.piece_ms = {k: 0.0 for k in PIECES}
        self.piece_n = {k: 0 for k in PIECES}

    def time_only(self, pieces):
        """Keep the in-graph timing events of `pieces` only and capture the
        trial graphs again now (each event is a graph node that also breaks
        the programmatic launch overlap of the kernels around it, ~10% of a
        trial for all pieces).  Call between iterations, outside a timed
        window; the engine's lazy resources are initialised by then, so the
        graphs are captured without a warm-up run."""
        self.reset_piece_times(pieces)
        self.piece_record = set(pieces)
        if not self.use_graphs or not self.graphs:
            return
        torch.cuda.synchronize(self.dev)
        # the old graphs keep the shared memory pool alive until the new ones
        # are captured into it
        old = (self.graphs, self.graph_exec, self.graph_kernels)
        self.graphs, self.graph_exec, self.graph_kernels = {}, {}, {}
        for q in range(NSLOT):
            for head in (False, True):
                self._graph(q, head, warm=False)
        torch.cuda.synchronize(self.dev)
        del old

    def piece_means(self):
        """Mean device ms per trial of each timed piece."""
        return {k: self.piece_ms[k] / self.piece_n[k] for k in PIECES if self.piece_n[k]}

    def evaluate(self, q):
        """HPWL and (overflow, max density) of V[q] into the parity-q metric buffers,
        for a position set from outside the trial kernel."""
        dc = self.data
        v = self.V[q]
        C.hpwl_lanes(self.xy(v), self.group_deg, self.group_base, self.group_net, self.ln_node, self.ln_offx,
                     self.ln_offy, dc.net_weights, dc.net_mask_all, self.H[q])
        self._density(v, 0, self.omap)
        C.density_overflow_into(self.omap, self.ovf_target, self.ovf_area, self.O[q])

    def move_boundary(self, v):
        d = self.design
        C.move_boundary_forward(v, self.data.node_size_x, self.data.node_size_y, float(d.xl), float(d.yl),
                                float(d.xh), float(d.yh), d.num_movable_nodes, d.num_filler_nodes)
        self.pack(v)
        for q in range(NSLOT):
            if v.data_ptr() == self.V[q].data_ptr():
                self.evaluate(q)

    # ---------------------------------------------------------------- setup
    def _plain_objective(self):
        """Set-up evaluations use the model's density factor without the
        quadratic penalty; the next step refreshes the loop's values."""
        self._quad_c = 0.0
        self.factor_quad.copy_(torch.tensor([float(self.model.density_factor), 0.0], dtype=torch.float32))
        self.graph_key = None

    def initial_learning_rate(self, lr):
        """|x0 - x1| / |g0 - g1| after x1 = x0 - lr g0 (PlaceObj.estimate_initial_learning_rate)."""
        v0, g0, g1, x1 = self.V[0], self.G[0], self.G[1], self.V[1]
        self._plain_objective()
        self.pack(v0)
        self.obj_and_raw_grad(v0, g0)
        self.precondition(g0, v0, g0, v0)
        torch.sub(v0, g0, alpha=lr, out=x1)
        self.pack(x1)
        self.obj_and_raw_grad(x1, g1)
        self.precondition(g1, v0, g0, x1)
        return float((torch.dist(v0.double(), x1.double()) / torch.dist(g0.double(), g1.double())).item())

    def initialize_density_weight(self):
        """lambda0 = density_weight * |grad WL|_1 / |grad D|_1 (PlaceObj.initialize_density_weight)."""
        v = self.V[self.slot]
        self.wirelength(v)
        self.wl_grad_into(self.tmp, False)
        wl_norm = self.tmp.double().abs().sum()
        ex, ey, energy = self.density_energy(v)
        self.density_grad_into(v, ex, ey, self.one, self.tmp)
        d_norm = self.tmp.double().abs().sum()
        self.model.init_density = energy.float().clone()
        m = self.model
        m.density_weight = (self.params.density_weight * wl_norm / d_norm).to(torch.float32).reshape(1)
        m.density_weight_grad_precond = torch.where(m.init_density > 0, 1 / m.init_density, m.init_density)
        m.quad_penalty_coeff = m.density_quad_coeff / 2 * m.density_weight_grad_precond

    def start_optimizer(self, lr):
        """First optimizer step's set-up: g_k at v_k, g_k_1 at v_k - lr g_k, alpha_k."""
        p = self.slot
        v, g, u = self.V[p], self.G[p], self.U[p]
        self._plain_objective()
        self.obj_and_raw_grad(v, g)
        self.precondition(g, v, g, v)
        u.copy_(v)
        x1, g1 = self.V[(p + 1) % NSLOT], self.G[(p + 1) % NSLOT]
        torch.sub(v, g, alpha=lr, out=x1)
        self.pack(x1)
        self.obj_and_raw_grad(x1, g1)
        self.precondition(g1, v, g, x1)
        alpha = float((torch.dist(v.double(), x1.double()) / torch.dist(g.double(), g1.double())).item())
        C.nesterov_init(self.S[p], alpha)
        # iteration 0's density weight and gamma come from the model (the set-up
        # above); later iterations' from dp_iteration_head
        m = self.model
        self.weights[p].copy_(torch.cat([m.density_weight.reshape(1).float(), m.gamma.reshape(1).float(),
                                         (1.0 / m.gamma.reshape(1)).float()]))
        self.sched[p].zero_()
        self.enqueued = None
        return alpha

    def sync_model(self):
        """Copy the current iteration's density weight and gamma (kept on the
        device by the trial graphs) into the model's tensors."""
        m, w = self.model, self.weights[self.slot]
        with torch.no_grad():
            m.density_weight.copy_(w[0:1].reshape(m.density_weight.shape))
            m.gamma.copy_(w[1].reshape(m.gamma.shape))

    # ---------------------------------------------------------------- iteration
    def _trial(self, s, head=False):
        """One Nesterov trial from slot s into slot s + 1.  head: the first trial
        of an iteration k >= 1, preceded by the loop's between-iteration work on
        the device (advance, density weight, gamma from slot s - 1)."""
        t = (s + 1) % NSLOT
        self._mark_slot = s
        gate = self.gate if self.use_graphs else None
        if head:
            r = (s - 1) % NSLOT
            C.iteration_head(self.S[r], self.S[s], self.sched[r], self.sched[s], self.H[r][0:1], self.O[r][0:1],
                             self.weights[r], self.weights[s], *self.head_scalars, gate=gate)
        elif gate is not None:
            C.trial_gate(gate)
        v, g = self.V[s], self.G[s]
        vn, gn = self.V[t], self.G[t]
        st = self.S[s]
        self._mark("nesterov_trial", 0)
        self.nesterov_trial_only(s)
        self._mark("nesterov_trial", 1)
        energy = self.objective_and_step(v, g, vn, gn, s)
        # HPWL / overflow of v_k (computed when v_k was the trial point), then the trial's scalars
        C.trial_metrics(self.H[s], self.O[s], st, self.obj64, self.wl64, energy, self.metrics[s])

    def nesterov_trial_only(self, s):
        """The trial point from slot s into slot s + 1, and its visiting-order
        copy for the scatter (xyo_mode "trial": written by the trial kernel
        through inv_order; "gather": gathered through order after it)."""
        d = self.design
        t = (s + 1) % NSLOT
        scatter_write = self.xyo_mode == "trial"
        C.nesterov_trial(self.V[s], self.G[s], self.U[s], self.U[t], self.V[t], self.XY[t], self.S[s],
                         self.data.node_size_x, self.data.node_size_y, float(d.xl), float(d.yl), float(d.xh),
                         float(d.yh), d.num_movable_nodes, d.num_filler_nodes,
                         self.inv_order if scatter_write else None, self.XYO[t] if scatter_write else None)
        if self.xyo_mode == "gather":
            C.gather_order_xy(self.XY[t], self.order, self.order.numel(), self.XYO[t])

    def _body(self, s, head):
        # v_k was clamped into the die when it was produced (trial kernel, or
        # move_boundary + pack at the start / after a rollback), so the
        # reference's per-iteration move_boundary(pos) is the identity here,
        # and its evaluation (HPWL, overflow) was computed with it
        self._trial(s, head)
        # the metrics' read-back is part of the trial (a copy node in the graph)
        self.metrics_host[s].copy_(self.metrics[s], non_blocking=True)

    def _graph(self, s, head, warm=True):
        key = (s, head)
        g = self.graphs.get(key)
        if g is None:
            if warm:
                # warm-up on a side stream.  Only the head-less body of the
                # current slot may run here: it writes the next slot's buffers,
                # which hold nothing yet, and the slot's optimizer scalars, which
                # are restored.
                assert s == self.slot and not head, "graph warm-up must run the current slot without head"
                st = torch.cuda.Stream()
                st.wait_stream(torch.cuda.current_stream())
                with torch.cuda.stream(st):
                    saved = self.S[s].clone()
                    self._body(s, head)
                    self.S[s].copy_(saved)
                torch.cuda.current_stream().wait_stream(st)
            # captured on a side stream with capture_begin / capture_end (the
            # torch.cuda.graph context would also run gc and empty the
            # allocator cache, which costs a stall inside the GP loop)
            g = torch.cuda.CUDAGraph()
            before = C.launch_count()
            st = torch.cuda.Stream()
            st.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(st):
                g.capture_begin(pool=self.pool)
                C.set_trial_gate(self.gate)
                try:
                    self._body(s, head)
                finally:
                    C.set_trial_gate(None)
                    g.capture_end()
            torch.cuda.current_stream().wait_stream(st)
            self.graph_kernels[key] = C.launch_count() - before
            if self.pool is None:
                self.pool = g.pool()
            self.graphs[key] = g
            self.graph_exec[key] = g.raw_cuda_graph_exec()
        return g

    def _launch(self, s, head):
        """Enqueue one trial from slot s (graph replay) and the read-back of its
        metrics on the current stream."""
        if self.best_slot == (s + 1) % NSLOT:
            self.flush_best()  # the trial overwrites the best position's slot
        if self.use_graphs:
            self._graph(s, head)
            C.graph_launch(self.graph_exec[(s, head)], torch._C._cuda_getCurrentRawStream(self._dev_index))
            self.kernels_launched += self.graph_kernels[(s, head)]
        else:
            before = C.launch_count()
            self._body(s, head)
            self.kernels_launched += C.launch_count() - before
        if self.ready[s] is None:
            self.ready[s] = torch.cuda.Event()
        self.ready[s].record(self._current_stream())

    def _current_stream(self):
        """The current stream, looked up again only when its handle changed
        (torch.cuda.current_stream() costs ~15 us of host time per call)."""
        raw = torch._C._cuda_getCurrentRawStream(self._dev_index)
        if raw != self._stream_raw:
            self._stream_obj = torch.cuda.current_stream(self.dev)
            self._stream_raw = raw
        return self._stream_obj

    def _collect(self, s):
        """Wait for the last trial launched from slot s and return its metrics."""
        self.ready[s].synchronize()
        if self.piece_events is not None:
            self._collect_pieces(s)
        return self.metrics_host[s].numpy().copy()

    def _run(self, s, head=False):
        self._launch(s, head)
        return self._collect(s)

    def _enqueue_first(self, k, s):
        """Enqueue the first trial of iteration k (input slot s), with the
        visiting-order refresh that iteration starts with."""
        if self.refresh_due(k):
            self.refresh_order(self.V[s])
        self._launch(s, k > 0)
        self.enqueued = k

    def refresh_due(self, k):
        """Whether iteration k starts with a visiting-order refresh."""
        for until, every in self.sort_schedule:
            if k < until:
                return every > 0 and k % every == 0
        return self.sort_interval > 0 and k % self.sort_interval == 0

    def _check_graph_key(self):
        """Refresh the device copy of (density factor, quadratic penalty
        coefficient) when the GP loop changed them (no recapture needed); an
        iteration enqueued ahead with the old values is enqueued again."""
        m = self.model
        key = (float(m.density_factor), bool(m.quad_penalty))
        if key != self.graph_key:
            self._quad_c = float(m.quad_penalty_coeff.item()) if m.quad_penalty else 0.0
            self.factor_quad.copy_(torch.tensor([key[0], self._quad_c], dtype=torch.float32))
            self.graph_key = key
            self.enqueued = None

    def prepare_graphs(self):
        """Capture the trial graphs of every slot (first trial with the
        between-iteration head, and retry) up front, so no capture happens inside
        a timed or latency-sensitive window."""
        if not self.use_graphs:
            return
        self._check_graph_key()
        s = self.slot
        # one warm-up (current slot, no head) initialises every lazy resource;
        # the other graphs are captured without running
        self._graph(s, False)
        for q in range(NSLOT):
            for head in (False, True):
                self._graph(q, head, warm=False)

    def step(self):
        """One GP iteration: evaluation at v_k, then Nesterov trials until accepted
        (<= 10).  Returns (hpwl, overflow / total movable area, max_density, objective, trials)."""
        gen = self.step_gen()
        try:
            while True:
                next(gen)
        except StopIteration as stop:
            return stop.value

    def step_gen(self):
        """step() as a generator: it yields once, right after the iteration's
        first trial is enqueued, so a driver of several designs can enqueue theirs
        (on their own streams) before this one waits for its metrics.

        With speculation the first trial of iteration k+1 is enqueued behind
        iteration k's before the host waits: its head does on the device what the
        host loop does between iterations, so the GPU never waits for the host.
        It is enqueued again when iteration k needed a retry, or the host changed
        the density factor or the position after reading iteration k."""
        self._check_graph_key()
        if self.use_graphs and len(self.graphs) < 2 * NSLOT:
            self.prepare_graphs()
        s = self.slot
        k = self.iterations
        if self.enqueued != k:
            self._enqueue_first(k, s)
        if self.speculate:
            self._enqueue_first(k + 1, (s + 1) % NSLOT)
        yield
        mh = self._collect(s)
        hpwl, ovf, maxd = mh[M_HPWL], mh[M_OVF], mh[M_MAXD]
        trials = 1
        while mh[M_ACCEPT] == 0.0 and trials < 10:
            # the iteration enqueued ahead saw the rejection (its gate closed);
            # enqueue it again behind the retry
            self._launch(s, False)
            if self.speculate:
                self._enqueue_first(k + 1, (s + 1) % NSLOT)
            else:
                self.enqueued = None
            mh = self._collect(s)
            trials += 1
        if mh[M_ACCEPT] == 0.0:
            # out of trials: the loop moves on with the last one, so the next
            # iteration must run (not see a rejection)
            self.S[s][NS_ACCEPT].fill_(1.0)
            self.enqueued = None
        self.iterations = k + 1
        self.slot = (s + 1) % NSLOT
        self.trials += trials
        return (float(hpwl), float(ovf) / self.design.total_movable_node_area, float(maxd), float(mh[M_OBJ]), trials)

    @property
    def parity(self):
        """The current slot (the iteration's input buffers)."""
        return self.slot

    def next_slot(self, s):
        return (s + 1) % NSLOT

    def current_position(self):
        return self.V[self.slot]

    def mark_best(self, buf=None):
        """Record the current position as the best one.  It is copied into
        ``buf`` (allocated when None) on the stream right before a trial
        overwrites its slot, or by flush_best; returns ``buf``."""
        if buf is None:
            buf = torch.empty_like(self.V[self.slot])
        self.best_buf = buf
        self.best_slot = self.slot
        return buf

    def flush_best(self):
        """Complete a pending best-position copy (stream-ordered)."""
        if self.best_slot is not None:
            self.best_buf.copy_(self.V[self.best_slot])
            self.best_slot = None
        return self.best_buf

    # ---------------------------------------------------------------- checkpoint
    _STATE_LISTS = ("V", "U", "G", "XY", "XYO", "S", "sched", "weights", "H", "O", "metrics")
    _STATE_TENSORS = ("order", "rec4", "ratio_o", "inv_order", "factor_quad", "gate")

    def state_dict(self):
        """The optimizer and iteration state on the host: the three slots'
        positions, u, g (and their interleaved / visiting-order copies),
        optimizer scalars, lambda / gamma, schedule words and metric buffers,
        the visiting order and its records, and the counters.  The device is
        synchronised first, so an iteration enqueued ahead has finished."""
        self.flush_best()
        torch.cuda.synchronize(self.dev)
        sd = {k: [t.detach().cpu().clone() for t in getattr(self, k)] for k in self._STATE_LISTS}
        sd.update({k: getattr(self, k).detach().cpu().clone() for k in self._STATE_TENSORS})
        sd.update(slot=self.slot, iterations=self.iterations, trials=self.trials, quad_c=self._quad_c)
        return sd

    def load_state_dict(self, sd):
        """Restores state_dict() into this engine's own buffers (captured trial
        graphs keep pointing at them); the next step starts iteration
        sd["iterations"] from slot sd["slot"], enqueued afresh."""
        with torch.no_grad():
            for k in self._STATE_LISTS:
                for dst, src in zip(getattr(self, k), sd[k]):
                    dst.copy_(src)
            for k in self._STATE_TENSORS:
                getattr(self, k).copy_(sd[k])
        self.slot, self.iterations, self.trials = int(sd["slot"]), int(sd["iterations"]), int(sd["trials"])
        self._quad_c = float(sd["quad_c"])
        self.enqueued = None
        self.graph_key = None
        self.best_slot = None

    def set_position(self, t):
        """Overwrite v_k (divergence rollback), clamped into the die; an
        iteration enqueued ahead from the old v_k is enqueued again."""
        self.flush_best()
        v = self.V[self.slot]
        v.copy_(t)
        self.move_boundary(v)
        self.enqueued = None
