"""Ops adjacent to the hot path that run on every GP iteration.

Drop-ins for the reference modules (paths relative to dreamplace/ops):
``pin_pos/pin_pos.py`` (PinPos), ``hpwl/hpwl.py`` (HPWL),
``move_boundary/move_boundary.py`` (MoveBoundary),
``pin_weight_sum/pin_weight_sum.py`` (PinWeightSum) and
``density_map/density_map.py`` (DensityMap).  HPWL is accumulated in fp64
(``HPWL.forward_f64``); ``forward`` returns it rounded to float32 like the
reference's float sum.
"""
import torch
from torch import nn
from torch.autograd import Function

from ._native import C, require_cuda


def _i32(t):
    return t if t.dtype == torch.int32 else t.to(torch.int32)


class PinPosFunction(Function):
    @staticmethod
    def forward(ctx, pos, pin_offset_x, pin_offset_y, pin2node_map, flat_node2pin_map, flat_node2pin_start_map,
                num_physical_nodes):
        require_cuda(pos, "pos")
        ctx.pos = pos
        ctx.flat_node2pin_map = flat_node2pin_map
        ctx.flat_node2pin_start_map = flat_node2pin_start_map
        ctx.num_physical_nodes = num_physical_nodes
        return C.pin_pos_forward(pos.view(-1), pin_offset_x, pin_offset_y, pin2node_map)

    @staticmethod
    def backward(ctx, grad_pin_pos):
        out = C.pin_pos_backward(grad_pin_pos.contiguous(), ctx.pos, ctx.flat_node2pin_map,
                                 ctx.flat_node2pin_start_map, ctx.num_physical_nodes)
        return out, None, None, None, None, None, None


class PinPos(nn.Module):
    """pin_x = x[pin2node] + pin_offset_x (reference pin_pos/pin_pos.py:103-156)."""

    def __init__(self, pin_offset_x, pin_offset_y, pin2node_map, flat_node2pin_map, flat_node2pin_start_map,
                 num_physical_nodes, algorithm='node-by-node'):
        super().__init__()
        self.pin_offset_x = pin_offset_x
        self.pin_offset_y = pin_offset_y
        self.pin2node_map = _i32(pin2node_map)
        self.flat_node2pin_map = _i32(flat_node2pin_map)
        self.flat_node2pin_start_map = _i32(flat_node2pin_start_map)
        self.num_physical_nodes = num_physical_nodes
        self.algorithm = algorithm

    def forward(self, pos):
        return PinPosFunction.apply(pos, self.pin_offset_x, self.pin_offset_y, self.pin2node_map,
                                    self.flat_node2pin_map, self.flat_node2pin_start_map, self.num_physical_nodes)


class HPWL(nn.Module):
    """Half-perimeter wirelength, net-by-net (reference hpwl/hpwl.py:61-102)."""

    def __init__(self, flat_netpin=None, netpin_start=None, pin2net_map=None, net_weights=None, net_mask=None,
                 algorithm='net-by-net'):
        super().__init__()
        self.flat_netpin = _i32(flat_netpin)
        self.netpin_start = _i32(netpin_start)
        self.pin2net_map = pin2net_map
        self.net_weights = net_weights
        self.net_mask = net_mask
        self.algorithm = algorithm

    def forward_f64(self, pos):
        require_cuda(pos, "pos")
        return C.hpwl_forward(pos.view(-1), self.flat_netpin, self.netpin_start, self.net_weights, self.net_mask)

    def forward(self, pos):
        return self.forward_f64(pos)[0].float()


class MoveBoundary(object):
    """Clamp movable and filler cells into the die, in place (reference move_boundary/move_boundary.py)."""

    def __init__(self, node_size_x, node_size_y, xl, yl, xh, yh, num_movable_nodes, num_filler_nodes):
        self.node_size_x = node_size_x
        self.node_size_y = node_size_y
        self.xl, self.yl, self.xh, self.yh = xl, yl, xh, yh
        self.num_movable_nodes = num_movable_nodes
        self.num_filler_nodes = num_filler_nodes

    def forward(self, pos):
        require_cuda(pos, "pos")
        C.move_boundary_forward(pos.data.view(-1), self.node_size_x, self.node_size_y, float(self.xl),
                                float(self.yl), float(self.xh), float(self.yh), self.num_movable_nodes,
                                self.num_filler_nodes)
        return pos

    def __call__(self, pos):
        return self.forward(pos)


class PinWeightSum(nn.Module):
    """Sum of net weights over each node's pins (reference pin_weight_sum/pin_weight_sum.py)."""

    def __init__(self, flat_nodepin=None, nodepin_start=None, pin2net_map=None, num_nodes=None,
                 algorithm='node-by-node'):
        super().__init__()
        self.flat_nodepin = _i32(flat_nodepin)
        self.nodepin_start = _i32(nodepin_start)
        self.pin2net_map = _i32(pin2net_map)
        self.num_nodes = num_nodes
        self.algorithm = algorithm

    def forward(self, net_weights):
        require_cuda(net_weights, "net_weights")
        return C.pws_forward(net_weights, self.flat_nodepin, self.nodepin_start, self.pin2net_map, self.num_nodes)


class DensityMapFunction(Function):
    """Exact-overlap density of a node range; called as ``DensityMapFunction.forward(...)``
    without ctx (reference density_map/density_map.py:27-46)."""

    @staticmethod
    def forward(pos, node_size_x, node_size_y, initial_density_map, xl, yl, xh, yh, num_bins_x, num_bins_y,
                range_begin, range_end, deterministic_flag):
        require_cuda(pos, "pos")
        return C.density_map_exact(pos.view(-1), node_size_x, node_size_y, [int(range_begin), int(range_end)],
                                   initial_density_map, float(xl), float(yl), float(xh), float(yh),
                                   int(num_bins_x), int(num_bins_y), int(bool(deterministic_flag)))


class DensityMap(object):
    """Exact density map of node ranges (reference density_map/density_map.py:49-113)."""

    def __init__(self, node_size_x, node_size_y, xl, yl, xh, yh, num_bins_x, num_bins_y, range_list,
                 deterministic_flag, initial_density_map=None):
        self.node_size_x = node_size_x
        self.node_size_y = node_size_y
        self.xl, self.yl, self.xh, self.yh = xl, yl, xh, yh
        self.num_bins_x = num_bins_x
        self.num_bins_y = num_bins_y
        self.range_list = range_list
        self.deterministic_flag = deterministic_flag
        self.initial_density_map = initial_density_map

    def forward(self, pos):
        if self.initial_density_map is None:
            self.initial_density_map = torch.zeros(self.num_bins_x, self.num_bins_y, dtype=pos.dtype,
                                                   device=pos.device)
        density_map = self.initial_density_map
        for r in self.range_list:
            if r[0] < r[1]:
                density_map = DensityMapFunction.forward(pos, self.node_size_x, self.node_size_y, density_map,
                                                         self.xl, self.yl, self.xh, self.yh, self.num_bins_x,
                                                         self.num_bins_y, r[0], r[1], self.deterministic_flag)
        return density_map
