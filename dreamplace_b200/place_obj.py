"""Placement objective on the device: data collection, ops and PlaceObj.

Mirrors the reference's ``dreamplace/BasicPlace.py`` (PlaceDataCollection,
op builders) and ``dreamplace/PlaceObj.py`` (objective WL + lambda*D,
PreconditionOp, density-weight and gamma schedules) for the default flow
(no fence regions, no routability / timing options).  Scalars that the
reference reads back with ``.item()`` inside the objective (lambda, gamma)
stay on the device here, so an evaluation issues no host synchronisation.
"""
import logging
import math

import numpy as np
import torch
from torch import nn

from . import electric_potential as ep_mod
from .placement_ops import HPWL, MoveBoundary, PinPos, PinWeightSum
from .weighted_average_wirelength import WeightedAverageWirelength

logger = logging.getLogger(__name__)


class PlaceDataCollection(object):
    """Device tensors of a design (reference dreamplace/BasicPlace.py:38-220)."""

    def __init__(self, pos, params, design, device):
        self.device = device
        self.pos = pos
        d = design
        t = lambda a, dt=None: torch.from_numpy(np.ascontiguousarray(a)).to(device if dt is None else device,  # noqa: E731
                                                                           dtype=dt)
        with torch.no_grad():
            self.node_size_x = t(d.node_size_x)
            self.node_size_y = t(d.node_size_y)
            self.pin_offset_x = t(d.pin_offset_x)
            self.pin_offset_y = t(d.pin_offset_y)
            self.target_density = torch.tensor(d.target_density, dtype=torch.float32, device=device)
            self.node_areas = self.node_size_x * self.node_size_y
            self.pin2node_map = t(d.pin2node_map.astype(np.int32))
            self.flat_node2pin_map = t(d.flat_node2pin_map.astype(np.int32))
            self.flat_node2pin_start_map = t(d.flat_node2pin_start_map.astype(np.int32))
            self.pin2net_map = t(d.pin2net_map.astype(np.int32))
            self.flat_net2pin_map = t(d.flat_net2pin_map.astype(np.int32))
            self.flat_net2pin_start_map = t(d.flat_net2pin_start_map.astype(np.int32))
            self.net_weights = t(d.net_weights)
            deg = np.diff(d.flat_net2pin_start_map)
            self.net_mask_all = t((deg >= 2).astype(np.uint8))
            self.net_mask_ignore_large_degrees = t(((deg >= 2) & (deg < params.ignore_net_degree)).astype(np.uint8))
            self.pin_mask_ignore_fixed_macros = self.pin2node_map >= d.num_movable_nodes
            # ascending-width order of movable cells (reference BasicPlace.py:186-188)
            _, order = torch.sort(self.node_size_x[:d.num_movable_nodes], stable=True)
            self.sorted_node_map = order.to(torch.int32)
            if d.target_density < 1:
                self.movable_macro_mask = t(d.movable_macro_mask)
            else:
                self.movable_macro_mask = None

    def bin_center_x_padded(self, design, padding, num_bins_x):
        bs = (design.xh - design.xl) / num_bins_x
        xl, xh = design.xl - padding * bs, design.xh + padding * bs
        return torch.from_numpy(design.bin_centers(xl, xh, bs)).to(self.device)

    def bin_center_y_padded(self, design, padding, num_bins_y):
        bs = (design.yh - design.yl) / num_bins_y
        yl, yh = design.yl - padding * bs, design.yh + padding * bs
        return torch.from_numpy(design.bin_centers(yl, yh, bs)).to(self.device)


class PlaceOpCollection(object):
    pass


def build_ops(params, design, data):
    """Adjacent ops (reference dreamplace/BasicPlace.py:444-529)."""
    ops = PlaceOpCollection()
    ops.pin_pos_op = PinPos(data.pin_offset_x, data.pin_offset_y, data.pin2node_map, data.flat_node2pin_map,
                            data.flat_node2pin_start_map, design.num_physical_nodes)
    ops.move_boundary_op = MoveBoundary(data.node_size_x, data.node_size_y, design.xl, design.yl, design.xh,
                                        design.yh, design.num_movable_nodes, design.num_filler_nodes)
    hpwl = HPWL(data.flat_net2pin_map, data.flat_net2pin_start_map, data.pin2net_map, data.net_weights,
                data.net_mask_all)
    ops.hpwl_op = lambda pos: hpwl(ops.pin_pos_op(pos))
    ops.hpwl_f64_op = lambda pos: hpwl.forward_f64(ops.pin_pos_op(pos))
    ops.pws_op = PinWeightSum(data.flat_node2pin_map, data.flat_node2pin_start_map, data.pin2net_map,
                              design.num_nodes)
    return ops


class PreconditionOp(object):
    """grad /= max(1, pws + alpha*lambda*area) (reference dreamplace/PlaceObj.py:37-132).
    The pin-weight sum depends only on the net weights, so it is computed once."""

    def __init__(self, design, data, ops):
        self.design = design
        self.data = data
        self.ops = ops
        self.alpha = 1.0
        self.iteration = 0
        self._pws = None

    def set_overflow(self, overflow):
        pass

    def __call__(self, grad, density_weight, update_mask=None, fix_nodes_mask=None):
        with torch.no_grad():
            if self._pws is None:
                self._pws = self.ops.pws_op(self.data.net_weights)
            precond = self._pws + self.alpha * density_weight * self.data.node_areas
            precond.clamp_(min=1.0)
            n = self.design.num_nodes
            grad.view(2, n).div_(precond)
            self.iteration += 1
        return grad


class PlaceObj(nn.Module):
    """Objective WL(pin_pos(pos)) + lambda * D(pos) (reference dreamplace/PlaceObj.py:136-1153)."""

    def __init__(self, density_weight, params, design, data, ops, global_place_params):
        super().__init__()
        self.density_quad_coeff = 2000
        self.init_density = None
        self.density_factor = 1
        self.quad_penalty = False
        self.update_mask = None
        self.fix_nodes_mask = None
        self.params = params
        self.design = design
        self.data = data
        self.ops = ops
        self.gp = global_place_params
        dev = data.pos[0].device
        self.density_weight = torch.tensor([density_weight], dtype=torch.float32, device=dev)
        nbx = global_place_params.get("num_bins_x", 0)
        nby = global_place_params.get("num_bins_y", 0)
        self.num_bins_x = nbx if nbx > 1 else design.num_bins_x
        self.num_bins_y = nby if nby > 1 else design.num_bins_y
        self.bin_size_x = (design.xh - design.xl) / self.num_bins_x
        self.bin_size_y = (design.yh - design.yl) / self.num_bins_y
        self.gamma = torch.tensor(10 * self.base_gamma(params, design), dtype=torch.float32, device=dev)
        self.ops.wirelength_op, self.ops.update_gamma_op = self.build_weighted_average_wl(params, design, data,
                                                                                         ops.pin_pos_op)
        self.ops.density_overflow_op = self.build_electric_overflow(params, design, data)
        self.ops.density_op = self.build_electric_potential(params, design, data)
        self.ops.update_density_weight_op = self.build_update_density_weight(params, design)
        self.ops.precondition_op = PreconditionOp(design, data, ops)
        self.ops.noise_op = self.build_noise(params, design, data)
        self.Lgamma_iteration = global_place_params["iteration"]
        self.Llambda_density_weight_iteration = global_place_params.get("Llambda_density_weight_iteration", 1)
        self.Lsub_iteration = global_place_params.get("Lsub_iteration", 1)

    # --- objective -------------------------------------------------------------
    def obj_fn(self, pos):
        self.wirelength = self.ops.wirelength_op(pos)
        self.density = self.ops.density_op(pos)
        if self.init_density is None:
            self.init_density = self.density.data.clone()
            self.density_weight_grad_precond = torch.where(self.init_density > 0, 1 / self.init_density,
                                                           self.init_density)
            self.quad_penalty_coeff = self.density_quad_coeff / 2 * self.density_weight_grad_precond
        if self.quad_penalty:
            self.density = self.density * (1 + self.quad_penalty_coeff * self.density)
        lam = (self.density_factor * self.density_weight).reshape(())
        return self.wirelength + lam * self.density

    def obj_and_grad_fn(self, pos):
        if pos.grad is not None:
            pos.grad.zero_()
        obj = self.obj_fn(pos)
        if obj.requires_grad:
            obj.backward()
        self.ops.precondition_op(pos.grad, self.density_weight, self.update_mask, self.fix_nodes_mask)
        return obj, pos.grad

    def forward(self):
        return self.obj_fn(self.data.pos[0])

    def estimate_initial_learning_rate(self, x_k, lr):
        """|x_k - x_k_1| / |g_k - g_k_1| after a step of lr (reference PlaceObj.py:443-454)."""
        obj_k, g_k = self.obj_and_grad_fn(x_k)
        g_k = g_k.clone()
        x_k_1 = torch.autograd.Variable(x_k - lr * g_k, requires_grad=True)
        obj_k_1, g_k_1 = self.obj_and_grad_fn(x_k_1)
        return (x_k - x_k_1).norm(p=2) / (g_k - g_k_1).norm(p=2)

    # --- op builders -------------------------------------------------------------
    def build_weighted_average_wl(self, params, design, data, pin_pos_op):
        wl = WeightedAverageWirelength(flat_netpin=data.flat_net2pin_map, netpin_start=data.flat_net2pin_start_map,
                                       pin2net_map=data.pin2net_map, net_weights=data.net_weights,
                                       net_mask=data.net_mask_ignore_large_degrees,
                                       pin_mask=data.pin_mask_ignore_fixed_macros, gamma=self.gamma,
                                       algorithm='merged')
        base_gamma = self.base_gamma(params, design)

        def wirelength_op(pos):
            return wl(pin_pos_op(pos))

        def update_gamma_op(iteration, overflow):
            self.update_gamma(iteration, overflow, base_gamma)

        return wirelength_op, update_gamma_op

    def build_electric_overflow(self, params, design, data):
        return ep_mod.ElectricOverflow(
            node_size_x=data.node_size_x, node_size_y=data.node_size_y,
            bin_center_x=data.bin_center_x_padded(design, 0, self.num_bins_x),
            bin_center_y=data.bin_center_y_padded(design, 0, self.num_bins_y),
            target_density=design.target_density, xl=design.xl, yl=design.yl, xh=design.xh, yh=design.yh,
            bin_size_x=self.bin_size_x, bin_size_y=self.bin_size_y, num_movable_nodes=design.num_movable_nodes,
            num_terminals=design.num_terminals, num_filler_nodes=0, padding=0,
            deterministic_flag=params.deterministic_flag, sorted_node_map=data.sorted_node_map,
            movable_macro_mask=data.movable_macro_mask)

    def build_electric_potential(self, params, design, data):
        return ep_mod.ElectricPotential(
            node_size_x=data.node_size_x, node_size_y=data.node_size_y,
            bin_center_x=data.bin_center_x_padded(design, 0, self.num_bins_x),
            bin_center_y=data.bin_center_y_padded(design, 0, self.num_bins_y),
            target_density=design.target_density, xl=design.xl, yl=design.yl, xh=design.xh, yh=design.yh,
            bin_size_x=self.bin_size_x, bin_size_y=self.bin_size_y, num_movable_nodes=design.num_movable_nodes,
            num_terminals=design.num_terminals, num_filler_nodes=design.num_filler_nodes, padding=0,
            deterministic_flag=params.deterministic_flag, sorted_node_map=data.sorted_node_map,
            movable_macro_mask=data.movable_macro_mask, fast_mode=bool(params.RePlAce_skip_energy_flag),
            precision=params.dct_precision, recompute_field=bool(getattr(params, "recompute_field", 0)))

    def initialize_density_weight(self, params, design):
        """lambda0 = density_weight * |grad WL|_1 / |grad D|_1 (reference PlaceObj.py:767-825)."""
        pos = self.data.pos[0]
        wirelength = self.ops.wirelength_op(pos)
        if pos.grad is not None:
            pos.grad.zero_()
        wirelength.backward()
        wl_norm = pos.grad.norm(p=1)
        pos.grad.zero_()
        density = self.ops.density_op(pos)
        self.init_density = density.data.clone()
        density.backward()
        d_norm = pos.grad.norm(p=1)
        self.density_weight = (params.density_weight * wl_norm / d_norm).reshape(1).to(torch.float32)
        return self.density_weight

    def build_update_density_weight(self, params, design):
        """RePlAce hpwl-mode multiplier (reference PlaceObj.py:827-851), branch-free on the device."""
        ref_hpwl = params.RePlAce_ref_hpwl
        lower, upper = params.RePlAce_LOWER_PCOF, params.RePlAce_UPPER_PCOF

        def update(cur_metric, prev_metric, iteration):
            with torch.no_grad():
                delta = (cur_metric.hpwl - prev_metric.hpwl).to(torch.float32)
                mu_dec = upper * max(math.pow(0.9999, float(iteration)), 0.98)
                mu_inc = upper * torch.pow(torch.tensor(upper, dtype=torch.float32, device=delta.device),
                                           -delta / ref_hpwl).clamp(min=lower, max=upper)
                mu = torch.where(delta < 0, torch.full_like(mu_inc, mu_dec), mu_inc)
                self.density_weight.mul_(mu)

        return update

    def base_gamma(self, params, design):
        return params.gamma * (self.bin_size_x + self.bin_size_y)

    def update_gamma(self, iteration, overflow, base_gamma):
        """gamma = base * 10^((overflow - 0.1)*20/9 - 1) (reference PlaceObj.py:901-915)."""
        coef = torch.pow(10, (overflow.to(torch.float32) - 0.1) * 20 / 9 - 1)
        self.gamma.data.copy_((base_gamma * coef).reshape(()))
        return True

    def build_noise(self, params, design, data):
        node_size = torch.cat([data.node_size_x, data.node_size_y], dim=0)

        def noise_op(pos, noise_ratio):
            with torch.no_grad():
                noise = torch.rand_like(pos)
                noise.sub_(0.5).mul_(node_size).mul_(noise_ratio)
                n = design.num_nodes
                noise[design.num_movable_nodes:n - design.num_filler_nodes].zero_()
                noise[n + design.num_movable_nodes:2 * n - design.num_filler_nodes].zero_()
                return pos.add_(noise)

        return noise_op
