"""Electrostatic density operator: scatter, Poisson solve, field gather.

Drop-in for the reference's ``dreamplace/ops/electric_potential/
electric_potential.py`` and ``electric_overflow.py``: same classes
(``ElectricDensityMapFunction``, ``ElectricOverflow``,
``ElectricPotentialFunction``, ``ElectricPotential``), constructor and
``forward`` signatures, with one added keyword, ``precision``, selecting the
Poisson-solve arithmetic (``fp32`` plain form, ``tf32``, ``bf16``,
``split_bf16``).

Forward (reference electric_potential.py:52-217):
  density = initial + scatter(movable, filler)           dp_density_map_f32 / _fx64
  rho = density / bin_area                                (in place, as the reference)
  a = DCT2(rho);  Ex = IDXST_IDCT(a wu/(wu^2+wv^2)/2);  Ey = IDCT_IDXST(a wv/(...)/2)
  energy = sum(IDCT2(a/(wu^2+wv^2)) * rho)                unless fast_mode
as four GEMM launches: rho C_N^T (transposed bf16/fp32 operand out), C_M T with
the spectral weights in the epilogue, the two right products batched in one
launch, and the two left products batched with the Ex/Ey stores.  The energy
is summed in the spectral domain by the second launch's epilogue,
  sum_xy rho IDCT2(a winv) = M N sum_uv w_u w_v winv_uv a_uv^2 (w_0 = 1/2),
so the potential map is never formed.
Backward: the hand-written adjoint ``-electric_force`` (reference :219-275).

The modules (``ElectricOverflow``, ``ElectricPotential``) keep a spatial
visiting order of their cells (``CellOrder``) and run the order-driven kernels
of the GP engine: the window scatter (block-local sort, 3 x 3-bin register
windows, shared-memory tiles) and the field gather over per-cell records,
whose force is put back in node order.  ``ElectricDensityMapFunction`` and
``ElectricPotentialFunction`` keep the reference's per-cell kernels for
callers of the Functions themselves.
With ``recompute_field`` the forward runs only the first two launches (the
energy) and keeps the normalised density map; the backward repeats the solve
for the field maps, so no field map is held between forward and backward.
"""
import logging
import math

import numpy as np
import torch
from torch import nn
from torch.autograd import Function

from ._native import C, precision_code, require_cuda
from .dct2_fft2 import (DCT2, EPI_ENERGY, EPI_SPECTRAL, EPI_STORE, EPI_STORE_T, IDCT2, IDCT_IDXST, IDXST_IDCT,
                        Operand, get_exact_expk, transform_matrices)

logger = logging.getLogger(__name__)


_SPECTRAL_CACHE = {}


def spectral_tables(M, N, wv_scale, device):
    """[3, M, N] fp32 tables (wx, wy, winv) of the spectral scaling (cached)."""
    key = (M, N, float(wv_scale), str(device))
    if key not in _SPECTRAL_CACHE:
        _SPECTRAL_CACHE[key] = C.spectral_weights(M, N, float(wv_scale), torch.device(device))
    return _SPECTRAL_CACHE[key]


def poisson_flops(M, N, precision):
    """Algorithmic GEMM flops of one poisson_solve: rho -> a (one 2-D transform)
    and a -> (Ex, Ey) (two 2-D transforms), x3 for split-BF16."""
    k = 3 if precision_code(precision) == 3 else 1
    return 3 * k * 2.0 * M * N * (M + N)


class PoissonWorkspace(object):
    """The intermediate operands and outputs of one M x N solve in one
    precision, allocated once: a caller that solves repeatedly on one stream
    (the GP engine, inside its captured trials) passes it to poisson_solve,
    which then allocates nothing.  The returned field maps and energy are the
    workspace's own buffers, overwritten by the next solve."""

    def __init__(self, M, N, prec, device):
        self.key = (M, N, prec)
        self.rho = Operand((M, N), prec, device) if prec != 0 else None
        self.t1 = Operand((N, M), prec, device)
        self.spec = [Operand((M, N), prec, device) for _ in range(2)]
        self.us = [Operand((N, M), prec, device) for _ in range(2)]
        self.ex = torch.empty(M, N, dtype=torch.float32, device=device)
        self.ey = torch.empty(M, N, dtype=torch.float32, device=device)
        self.energy = torch.zeros(1, dtype=torch.float64, device=device)

    def check(self, M, N, prec):
        if self.key != (M, N, prec):
            raise ValueError("poisson workspace is for %s, not %s" % (self.key, (M, N, prec)))
        return self


def _poisson_spectral(rho, bin_size_x, bin_size_y, prec, energy, rho_scale=1.0, ws=None):
    """G1 and G2 of the solve: the two spectral operands a*wx, a*wy [M, N];
    when ``energy`` (f64[1]) is given the G2 epilogue adds the energy to it.
    The solve runs on rho * rho_scale (the scale is G1's alpha).  With a
    PoissonWorkspace ``ws`` the operands are the workspace's."""
    M, N = rho.shape
    dev = rho.device
    cM = transform_matrices(M, prec, dev)[0]
    cN = transform_matrices(N, prec, dev)[0]
    # G1: T1^T = (rho C_N^T)^T, [N, M]
    t1 = ws.t1 if ws is not None else Operand((N, M), prec, dev)
    g1 = dict(lda=N, ldb=N, epilogue=EPI_STORE_T, alpha=float(rho_scale), ldc=M)
    if prec == 0:
        g1["a_hi"] = rho
    elif ws is not None:
        ws.rho.fill(rho).as_a(g1)
    else:
        Operand.from_tensor(rho, prec).as_a(g1)
    cN.as_b(g1)
    t1.as_out_t(g1)
    C.transform_gemm(prec, M, N, N, [g1])
    # G2: a = 4/(MN) C_M T1 -> spectral operands a*wx, a*wy  [M, N]; the energy
    # sum(rho * IDCT2(a*winv)) = MN sum w_u w_v winv a^2 is summed in the same
    # epilogue, so the potential map is never formed
    spec = ws.spec if ws is not None else [Operand((M, N), prec, dev) for _ in range(2)]
    g2 = dict(lda=M, ldb=M, epilogue=EPI_SPECTRAL, alpha=4.0 / (M * N), ldc=N,
              wv_scale=float(bin_size_x / bin_size_y),
              spec_weights=spectral_tables(M, N, float(bin_size_x / bin_size_y), dev))
    if energy is not None:
        g2["energy"] = energy
    cM.as_a(g2)
    t1.as_b(g2)
    for i, s in enumerate(spec):
        if s.f32 is not None:
            g2["sp%d_f32" % i] = s.f32
        else:
            g2["sp%d_hi" % i] = s.hi
            g2["sp%d_lo" % i] = s.lo
    C.transform_gemm(prec, M, N, M, [g2])
    return spec


def poisson_energy(rho, bin_size_x, bin_size_y, precision):
    """Energy (f64[1]) of a normalised density map without the field maps:
    G1 and G2 only (two launches)."""
    energy = torch.zeros(1, dtype=torch.float64, device=rho.device)
    _poisson_spectral(rho, bin_size_x, bin_size_y, precision_code(precision), energy)
    return energy


def poisson_solve(rho, bin_size_x, bin_size_y, precision, fast_mode=False, rho_scale=1.0, ws=None):
    """Field maps and energy of a normalised density map ``rho`` [M, N] (fp32).

    Returns (field_map_x, field_map_y, energy_f64[1]); energy is zero when
    ``fast_mode``.  Four GEMM launches, see the module docstring.  With
    rho_scale the map is normalised inside the first GEMM (its alpha): a
    density map and rho_scale = 1 / bin area give the solve of rho.  With a
    PoissonWorkspace ``ws`` nothing is allocated and the results are the
    workspace's buffers."""
    prec = precision_code(precision)
    M, N = rho.shape
    dev = rho.device
    _, chM, shM = transform_matrices(M, prec, dev)
    _, chN, shN = transform_matrices(N, prec, dev)
    if ws is not None:
        ws.check(M, N, prec)
        energy = ws.energy
        C.zero_(energy)
    else:
        energy = torch.zeros(1, dtype=torch.float64, device=dev)
    spec = _poisson_spectral(rho, bin_size_x, bin_size_y, prec, None if fast_mode else energy, rho_scale, ws)
    # G3: U^T = (A R^T)^T for the x field (R = Ch_N) and the y field (Sh_N)
    rights = [chN, shN]
    us = ws.us if ws is not None else [Operand((N, M), prec, dev) for _ in spec]
    g3 = []
    for s, r, u in zip(spec, rights, us):
        d = dict(lda=N, ldb=N, epilogue=EPI_STORE_T, alpha=1.0, ldc=M)
        s.as_a(d)
        r.as_b(d)
        u.as_out_t(d)
        g3.append(d)
    C.transform_gemm(prec, M, N, N, g3)
    # G4: Ex = 4 Sh_M Ux, Ey = 4 Ch_M Uy
    if ws is not None:
        ex, ey = ws.ex, ws.ey
    else:
        ex = torch.empty(M, N, dtype=torch.float32, device=dev)
        ey = torch.empty(M, N, dtype=torch.float32, device=dev)
    g4 = [shM.as_a(us[0].as_b(dict(lda=M, ldb=M, epilogue=EPI_STORE, alpha=4.0, ldc=N, out_f32=ex))),
          chM.as_a(us[1].as_b(dict(lda=M, ldb=M, epilogue=EPI_STORE, alpha=4.0, ldc=N, out_f32=ey)))]
    C.transform_gemm(prec, M, N, M, g4)
    return ex, ey, energy


class ElectricDensityMapFunction(Function):
    """Density map of movable + filler cells on top of the fixed-cell map.

    Called directly (``ElectricDensityMapFunction.forward(...)``, no ctx) as in
    the reference electric_overflow.py:57-114."""

    @staticmethod
    def forward(pos, node_size_x_clamped, node_size_y_clamped, offset_x, offset_y, ratio, bin_center_x,
                bin_center_y, initial_density_map, target_density, xl, yl, xh, yh, bin_size_x, bin_size_y,
                num_movable_nodes, num_filler_nodes, padding, padding_mask, num_bins_x, num_bins_y,
                num_movable_impacted_bins_x, num_movable_impacted_bins_y, num_filler_impacted_bins_x,
                num_filler_impacted_bins_y, deterministic_flag, sorted_node_map):
        require_cuda(pos, "pos")
        output = C.density_map(pos.view(pos.numel()), node_size_x_clamped, node_size_y_clamped, offset_x,
                               offset_y, ratio, bin_center_x, bin_center_y, initial_density_map,
                               float(target_density), float(xl), float(yl), float(xh), float(yh),
                               float(bin_size_x), float(bin_size_y), int(num_movable_nodes),
                               int(num_filler_nodes), int(padding), int(num_bins_x), int(num_bins_y),
                               int(num_movable_impacted_bins_x), int(num_movable_impacted_bins_y),
                               int(num_filler_impacted_bins_x), int(num_filler_impacted_bins_y),
                               int(bool(deterministic_flag)), sorted_node_map)
        density_map = output.view([num_bins_x, num_bins_y])
        if padding > 0:
            density_map.masked_fill_(padding_mask, target_density * bin_size_x * bin_size_y)
        return density_map


class CellOrder(object):
    """Spatial visiting order of a module's scattered cells (movable, then
    fillers) for the order-driven scatter and field gather: the cells bucketed
    by the bin where their stretched footprint starts (dp_order_cells_by_bin)
    and their records (stretched sizes, offsets, ratio) in that order.  The
    order is refreshed every ``interval`` calls of ``positions``; any order is
    valid (fixed-point maps do not depend on it), a fresh one keeps each
    scatter block's cells on a compact patch of bins.  A refresh allocates new
    tensors, so a backward still holding the previous order is unaffected."""

    def __init__(self, op, num_filler_nodes, interval=50):
        self.op = op
        self.count = op.num_movable_nodes + num_filler_nodes
        self.num_filler = num_filler_nodes
        self.interval = int(interval)
        self.calls = 0
        self.order = self.rec4 = self.ratio_o = None
        self._scratch = None

    def _refresh(self, pos):
        op = self.op
        dev = pos.device
        nm, nf = op.num_movable_nodes, self.num_filler
        if self._scratch is None:
            nbytes = C.order_cells_scratch_bytes(nm, nf, op.num_bins_x, op.num_bins_y)
            self._scratch = torch.empty((nbytes + 3) // 4, dtype=torch.int32, device=dev)
        order = torch.empty(self.count, dtype=torch.int32, device=dev)
        C.order_cells_by_bin(pos, op.offset_x, op.offset_y, nm, nf, float(op.xl), float(op.yl),
                             float(op.bin_size_x), float(op.bin_size_y), op.num_bins_x, op.num_bins_y,
                             self._scratch, order)
        rec4 = torch.empty(4 * self.count, dtype=torch.float32, device=dev)
        ratio_o = torch.empty(self.count, dtype=torch.float32, device=dev)
        C.build_cell_records(op.node_size_x_clamped, op.node_size_y_clamped, op.offset_x, op.offset_y, op.ratio,
                             order, self.count, rec4, ratio_o, None)
        self.order, self.rec4, self.ratio_o = order, rec4, ratio_o

    def positions(self, pos):
        """The cells' positions in visiting order (interleaved), refreshing the
        order when due; returns (xy_o, order, rec4, ratio_o)."""
        if self.order is None or (self.interval > 0 and self.calls % self.interval == 0):
            self._refresh(pos)
        self.calls += 1
        xy_o = torch.empty(2 * self.count, dtype=torch.float32, device=pos.device)
        C.gather_order_pos(pos, self.order, self.count, xy_o)
        return xy_o, self.order, self.rec4, self.ratio_o


class ElectricOverflow(nn.Module):
    """Overflow / max-density evaluation (reference electric_overflow.py:117-278)."""

    def __init__(self, node_size_x, node_size_y, bin_center_x, bin_center_y, target_density, xl, yl, xh, yh,
                 bin_size_x, bin_size_y, num_movable_nodes, num_terminals, num_filler_nodes, padding,
                 deterministic_flag, sorted_node_map, movable_macro_mask=None):
        super().__init__()
        self.node_size_x = node_size_x
        self.node_size_y = node_size_y
        self.bin_center_x = bin_center_x
        self.bin_center_y = bin_center_y
        self.target_density = target_density
        self.xl, self.yl, self.xh, self.yh = xl, yl, xh, yh
        self.bin_size_x = bin_size_x
        self.bin_size_y = bin_size_y
        self.num_movable_nodes = num_movable_nodes
        self.num_terminals = num_terminals
        self.num_filler_nodes = num_filler_nodes
        self.padding = padding
        self.sorted_node_map = sorted_node_map
        self.movable_macro_mask = movable_macro_mask
        self.deterministic_flag = deterministic_flag
        self.reset()

    def reset(self):
        """Stretched sizes, offsets and area ratios (reference electric_overflow.py:162-227)."""
        sqrt2 = math.sqrt(2)
        self.node_size_x_clamped = self.node_size_x.clamp(min=self.bin_size_x * sqrt2)
        self.offset_x = (self.node_size_x - self.node_size_x_clamped).mul(0.5)
        self.node_size_y_clamped = self.node_size_y.clamp(min=self.bin_size_y * sqrt2)
        self.offset_y = (self.node_size_y - self.node_size_y_clamped).mul(0.5)
        node_areas = self.node_size_x * self.node_size_y
        self.ratio = node_areas / (self.node_size_x_clamped * self.node_size_y_clamped)
        self.num_movable_macros = 0
        if self.target_density < 1 and self.movable_macro_mask is not None:
            self.num_movable_macros = int(self.movable_macro_mask.sum().item())
            self.ratio[:self.num_movable_nodes][self.movable_macro_mask] = self.target_density
        self.num_bins_x = int(round((self.xh - self.xl) / self.bin_size_x))
        self.num_bins_y = int(round((self.yh - self.yl) / self.bin_size_y))
        nm, nf = self.num_movable_nodes, self.num_filler_nodes
        if nm:
            self.num_movable_impacted_bins_x = int(math.ceil(min(
                (float(self.node_size_x[:nm].max()) + 2 * sqrt2 * self.bin_size_x) / self.bin_size_x, self.num_bins_x)))
            self.num_movable_impacted_bins_y = int(math.ceil(min(
                (float(self.node_size_y[:nm].max()) + 2 * sqrt2 * self.bin_size_y) / self.bin_size_y, self.num_bins_y)))
        else:
            self.num_movable_impacted_bins_x = self.num_movable_impacted_bins_y = 0
        if nf:
            self.num_filler_impacted_bins_x = int(math.ceil(min(
                (float(self.node_size_x[-nf:].max()) + 2 * sqrt2 * self.bin_size_x) / self.bin_size_x, self.num_bins_x)))
            self.num_filler_impacted_bins_y = int(math.ceil(min(
                (float(self.node_size_y[-nf:].max()) + 2 * sqrt2 * self.bin_size_y) / self.bin_size_y, self.num_bins_y)))
        else:
            self.num_filler_impacted_bins_x = self.num_filler_impacted_bins_y = 0
        dev = self.node_size_x.device
        self.padding_mask = torch.zeros(self.num_bins_x, self.num_bins_y, dtype=torch.bool, device=dev)
        if self.padding > 0:
            self.padding_mask.fill_(True)
            self.padding_mask[self.padding:self.num_bins_x - self.padding,
                              self.padding:self.num_bins_y - self.padding] = False
        self.initial_density_map = None
        self._orders = {}
        self._fixed_scratch = None

    def cell_order(self, num_filler_nodes):
        """The visiting order of the movable cells and num_filler_nodes fillers."""
        o = self._orders.get(num_filler_nodes)
        if o is None:
            o = self._orders[num_filler_nodes] = CellOrder(self, num_filler_nodes)
        return o

    def fixed_scratch(self, device):
        """The int64 accumulation map of the deterministic scatter (one per module)."""
        if self._fixed_scratch is None:
            self._fixed_scratch = torch.empty(self.num_bins_x * self.num_bins_y, dtype=torch.int64, device=device)
        return self._fixed_scratch

    def ordered_density_map(self, pos, num_filler_nodes):
        """The density map of the movable cells and num_filler_nodes fillers on
        the initial map, by the order-driven scatter (window kernel, block-local
        sort, shared-memory tiles): the same map as ElectricDensityMapFunction
        (bit for bit in deterministic mode), with the padding bins filled.
        Returns (density_map [M, N], (xy_o, order, rec4, ratio_o))."""
        require_cuda(pos, "pos")
        cells = self.cell_order(num_filler_nodes).positions(pos.view(pos.numel()))
        xy_o, order, rec4, ratio_o = cells
        M, N = self.num_bins_x, self.num_bins_y
        det = int(bool(self.deterministic_flag))
        scratch = self.fixed_scratch(pos.device) if det else None
        geo = (float(self.xl), float(self.yl), float(self.xh), float(self.yh), float(self.bin_size_x),
               float(self.bin_size_y), M, N)
        out = torch.empty(M * N, dtype=torch.float32, device=pos.device)
        nm = self.num_movable_nodes
        count = nm + num_filler_nodes
        if num_filler_nodes > 0 and nm > 0:
            # movable cells block-sorted, fillers (about one per bin) not
            first = torch.empty_like(out)
            C.density_map_ordered_split(xy_o, rec4, ratio_o, nm, count, self.initial_density_map.view(-1), *geo, det,
                                        scratch, first, out, 1.0, 1.0, None)
        else:
            C.density_map_ordered_into(xy_o, rec4, ratio_o, count, self.initial_density_map.view(-1), *geo, det,
                                       scratch, out)
        density_map = out.view(M, N)
        if self.padding > 0:
            density_map.masked_fill_(self.padding_mask, self.target_density * self.bin_size_x * self.bin_size_y)
        return density_map, cells

    def compute_initial_density_map(self, pos):
        """Fixed-cell map ×target_density (reference electric_overflow.py:229-258)."""
        nm, nt = self.num_movable_nodes, self.num_terminals
        if nt == 0:
            nfx = nfy = 0
        else:
            nfx = int(math.ceil(min((float(self.node_size_x[nm:nm + nt].max()) + self.bin_size_x) / self.bin_size_x,
                                    self.num_bins_x)))
            nfy = int(math.ceil(min((float(self.node_size_y[nm:nm + nt].max()) + self.bin_size_y) / self.bin_size_y,
                                    self.num_bins_y)))
        self.initial_density_map = C.fixed_density_map(
            pos, self.node_size_x, self.node_size_y, self.bin_center_x, self.bin_center_y, float(self.xl),
            float(self.yl), float(self.xh), float(self.yh), float(self.bin_size_x), float(self.bin_size_y), nm, nt,
            self.num_bins_x, self.num_bins_y, nfx, nfy, int(bool(self.deterministic_flag)))
        self.initial_density_map.mul_(self.target_density)

    def _density_map(self, pos, num_filler_nodes):
        return ElectricDensityMapFunction.forward(
            pos, self.node_size_x_clamped, self.node_size_y_clamped, self.offset_x, self.offset_y, self.ratio,
            self.bin_center_x, self.bin_center_y, self.initial_density_map, self.target_density, self.xl,
            self.yl, self.xh, self.yh, self.bin_size_x, self.bin_size_y, self.num_movable_nodes,
            num_filler_nodes, self.padding, self.padding_mask, self.num_bins_x, self.num_bins_y,
            self.num_movable_impacted_bins_x, self.num_movable_impacted_bins_y,
            self.num_filler_impacted_bins_x, self.num_filler_impacted_bins_y, self.deterministic_flag,
            self.sorted_node_map)

    def overflow_f64(self, pos):
        """(overflow, max_density) accumulated in fp64, as a [2] float64 tensor."""
        if self.initial_density_map is None:
            self.compute_initial_density_map(pos)
        density_map, _ = self.ordered_density_map(pos, self.num_filler_nodes)
        bin_area = self.bin_size_x * self.bin_size_y
        return C.density_overflow(density_map, float(self.target_density * bin_area), float(bin_area))

    def forward(self, pos):
        out = self.overflow_f64(pos)
        return out[0:1].float(), out[1:2].float()


class ElectricPotentialFunction(Function):
    """Energy forward / electric-force backward (reference electric_potential.py:47-275)."""

    @staticmethod
    def forward(ctx, pos, node_size_x_clamped, node_size_y_clamped, offset_x, offset_y, ratio, bin_center_x,
                bin_center_y, initial_density_map, target_density, xl, yl, xh, yh, bin_size_x, bin_size_y,
                num_movable_nodes, num_filler_nodes, padding, padding_mask, num_bins_x, num_bins_y,
                num_movable_impacted_bins_x, num_movable_impacted_bins_y, num_filler_impacted_bins_x,
                num_filler_impacted_bins_y, deterministic_flag, sorted_node_map, exact_expkM=None,
                exact_expkN=None, inv_wu2_plus_wv2=None, wu_by_wu2_plus_wv2_half=None,
                wv_by_wu2_plus_wv2_half=None, dct2=None, idct2=None, idct_idxst=None, idxst_idct=None,
                fast_mode=True, precision="fp32", recompute_field=False):
        density_map = ElectricDensityMapFunction.forward(
            pos, node_size_x_clamped, node_size_y_clamped, offset_x, offset_y, ratio, bin_center_x,
            bin_center_y, initial_density_map, target_density, xl, yl, xh, yh, bin_size_x, bin_size_y,
            num_movable_nodes, num_filler_nodes, padding, padding_mask, num_bins_x, num_bins_y,
            num_movable_impacted_bins_x, num_movable_impacted_bins_y, num_filler_impacted_bins_x,
            num_filler_impacted_bins_y, deterministic_flag, sorted_node_map)
        ctx.args = (num_bins_x, num_bins_y, num_movable_impacted_bins_x, num_movable_impacted_bins_y,
                    num_filler_impacted_bins_x, num_filler_impacted_bins_y)
        ctx.node = (node_size_x_clamped, node_size_y_clamped, offset_x, offset_y, ratio, bin_center_x,
                    bin_center_y)
        ctx.geom = (xl, yl, xh, yh, bin_size_x, bin_size_y, num_movable_nodes, num_filler_nodes)
        ctx.deterministic_flag = deterministic_flag
        ctx.sorted_node_map = sorted_node_map
        ctx.pos = pos
        density_map.mul_(1.0 / (bin_size_x * bin_size_y))
        ctx.precision = precision
        ctx.density_map = density_map
        if recompute_field:
            # keep only rho; the backward recomputes the field maps
            energy = torch.zeros(1, dtype=torch.float64, device=pos.device) if fast_mode else \
                poisson_energy(density_map, bin_size_x, bin_size_y, precision)
            ctx.field_map_x = ctx.field_map_y = None
        else:
            ex, ey, energy = poisson_solve(density_map, bin_size_x, bin_size_y, precision, fast_mode)
            ctx.field_map_x = ex
            ctx.field_map_y = ey
        if fast_mode:
            return torch.zeros(1, dtype=pos.dtype, device=pos.device)
        return energy.to(pos.dtype).view([])

    @staticmethod
    def backward(ctx, grad_pos):
        nbx, nby, a, b, c, d = ctx.args
        sxc, syc, ox, oy, ratio, bcx, bcy = ctx.node
        xl, yl, xh, yh, bsx, bsy, nm, nf = ctx.geom
        g = grad_pos.reshape(1).to(torch.float32)
        fx, fy = ctx.field_map_x, ctx.field_map_y
        if fx is None:
            fx, fy, _ = poisson_solve(ctx.density_map, bsx, bsy, ctx.precision, True)
        output = C.electric_force(g, nbx, nby, a, b, c, d, fx.view([-1]), fy.view([-1]),
                                  ctx.pos, sxc, syc, ox, oy, ratio, bcx, bcy, float(xl), float(yl), float(xh),
                                  float(yh), float(bsx), float(bsy), int(nm), int(nf),
                                  int(bool(ctx.deterministic_flag)), ctx.sorted_node_map, -1.0)
        return (output,) + (None,) * 39


class ElectricPotentialOrderedFunction(Function):
    """ElectricPotentialFunction over a visiting order: the order-driven
    scatter in forward and the order-driven field gather in backward
    (dp_electric_force_ordered), whose force is put back in node order; the
    same results as ElectricPotentialFunction (bit for bit in deterministic
    mode)."""

    @staticmethod
    def forward(ctx, pos, op, precision, fast_mode, recompute_field):
        density_map, cells = op.ordered_density_map(pos, op.num_filler_nodes)
        bsx, bsy = op.bin_size_x, op.bin_size_y
        density_map.mul_(1.0 / (bsx * bsy))
        ctx.op, ctx.cells, ctx.precision = op, cells, precision
        ctx.num_nodes = pos.numel() // 2
        ctx.density_map = density_map
        if recompute_field:
            energy = torch.zeros(1, dtype=torch.float64, device=pos.device) if fast_mode else \
                poisson_energy(density_map, bsx, bsy, precision)
            ctx.field_map_x = ctx.field_map_y = None
        else:
            ex, ey, energy = poisson_solve(density_map, bsx, bsy, precision, fast_mode)
            ctx.field_map_x, ctx.field_map_y = ex, ey
        if fast_mode:
            return torch.zeros(1, dtype=pos.dtype, device=pos.device)
        return energy.to(pos.dtype).view([])

    @staticmethod
    def backward(ctx, grad_pos):
        op = ctx.op
        xy_o, order, rec4, ratio_o = ctx.cells
        count = order.numel()
        fx, fy = ctx.field_map_x, ctx.field_map_y
        if fx is None:
            fx, fy, _ = poisson_solve(ctx.density_map, op.bin_size_x, op.bin_size_y, ctx.precision, True)
        g = grad_pos.reshape(1).to(torch.float32)
        force_o = torch.empty(2 * count, dtype=torch.float32, device=g.device)
        C.electric_force_ordered(g, fx.view(-1), fy.view(-1), xy_o, rec4, ratio_o, count, float(op.xl), float(op.yl),
                                 float(op.bin_size_x), float(op.bin_size_y), op.num_bins_x, op.num_bins_y, -1.0,
                                 force_o)
        output = C.scatter_pairs_to_nodes(force_o, order, count, ctx.num_nodes)
        return output, None, None, None, None


class ElectricPotential(ElectricOverflow):
    """Electrostatic density penalty (reference electric_potential.py:278-553)."""

    def __init__(self, node_size_x, node_size_y, bin_center_x, bin_center_y, target_density, xl, yl, xh, yh,
                 bin_size_x, bin_size_y, num_movable_nodes, num_terminals, num_filler_nodes, padding,
                 deterministic_flag, sorted_node_map, movable_macro_mask=None, fast_mode=False, region_id=None,
                 fence_regions=None, node2fence_region_map=None, placedb=None, precision="fp32",
                 recompute_field=False):
        if region_id is not None or fence_regions is not None:
            raise NotImplementedError("fence-region electric fields are not supported by dreamplace_b200")
        super().__init__(node_size_x=node_size_x, node_size_y=node_size_y, bin_center_x=bin_center_x,
                         bin_center_y=bin_center_y, target_density=target_density, xl=xl, yl=yl, xh=xh, yh=yh,
                         bin_size_x=bin_size_x, bin_size_y=bin_size_y, num_movable_nodes=num_movable_nodes,
                         num_terminals=num_terminals, num_filler_nodes=num_filler_nodes, padding=padding,
                         deterministic_flag=deterministic_flag, sorted_node_map=sorted_node_map,
                         movable_macro_mask=movable_macro_mask)
        self.fast_mode = fast_mode
        self.precision = precision_code(precision)
        # True: the forward keeps only the normalised density map and the
        # backward recomputes the field maps (less memory held between the two)
        self.recompute_field = recompute_field
        self.region_id = None
        self.fence_regions = None

    def reset(self):
        super().reset()
        self.exact_expkM = self.exact_expkN = None
        self.dct2 = self.idct2 = self.idct_idxst = self.idxst_idct = None

    def forward(self, pos, mode="density"):
        assert mode in {"density", "overflow"}, "Only support density mode or overflow mode"
        if self.initial_density_map is None:
            self.compute_initial_density_map(pos)
            M, N = self.num_bins_x, self.num_bins_y
            self.exact_expkM = get_exact_expk(M, dtype=pos.dtype, device=pos.device)
            self.exact_expkN = get_exact_expk(N, dtype=pos.dtype, device=pos.device)
            self.dct2 = DCT2(self.exact_expkM, self.exact_expkN, self.precision)
            if not self.fast_mode:
                self.idct2 = IDCT2(self.exact_expkM, self.exact_expkN, self.precision)
            self.idct_idxst = IDCT_IDXST(self.exact_expkM, self.exact_expkN, self.precision)
            self.idxst_idct = IDXST_IDCT(self.exact_expkM, self.exact_expkN, self.precision)
        if mode == "density":
            return ElectricPotentialOrderedFunction.apply(pos, self, self.precision, self.fast_mode,
                                                          self.recompute_field)
        density_map, _ = self.ordered_density_map(pos, 0)
        bin_area = self.bin_size_x * self.bin_size_y
        out = C.density_overflow(density_map, float(self.target_density * bin_area), float(bin_area))
        return out[0].float(), out[1].float()
