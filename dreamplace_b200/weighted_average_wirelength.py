"""Weighted-average wirelength (drop-in for the reference's
``dreamplace/ops/weighted_average_wirelength/weighted_average_wirelength.py``).

``WeightedAverageWirelength(flat_netpin, netpin_start, pin2net_map, net_weights,
net_mask, pin_mask, gamma, algorithm)`` with ``.forward(pin_pos)``.  The
reference offers net-by-net, atomic and merged algorithms that compute the
same function; the global placer uses ``merged``
(dreamplace/PlaceObj.py:475), which is what runs here for every name: one
forward pass writes the per-pin gradient (``grad_intermediate``) and backward
only scales it by ``grad_out`` and the net weight and zeroes masked pins
(reference :160-213).  ``gamma`` is a tensor re-read on every call because
the placer updates it in place.

The module runs the lane-per-net kernel (``dp_wa_pins_forward``): on its first
call it plans the nets once, 32 nets of one degree per warp with their pins
stored transposed so that every pin load of a warp is one coalesced access,
and one warp per net above 8 pins.  The forward leaves the per-pin gradient
(times the net weight) in lane-slot order; the backward gathers it back to
the reference's pin layout.  ``WeightedAverageWirelengthMergedFunction`` keeps
the reference's one-thread-per-net shape for callers of the Function itself.
"""
import torch
from torch import nn
from torch.autograd import Function

from ._native import C, require_cuda

REDUCE_DOUBLES = 1280


class PinLanes(object):
    """The lane plan of a netlist (dp_plan_net_lanes) with the pin arrays in
    lane-slot order: ln_pin (pin id of each lane slot) and lane_of_pin."""

    def __init__(self, flat_netpin, netpin_start):
        dev = flat_netpin.device
        g_deg, g_base, g_net, l_slot = C.plan_net_lanes(netpin_start.to("cpu", torch.int32).contiguous(), None)
        self.group_deg, self.group_base, self.group_net = g_deg.to(dev), g_base.to(dev), g_net.to(dev)
        ls = l_slot.to(dev).long()
        real = ls >= 0
        pin = flat_netpin.long()[ls.clamp(min=0)]
        self.ln_pin = torch.where(real, pin, torch.zeros_like(pin)).to(torch.int32).contiguous()
        self.num_slots = ls.numel()
        self.lane_of_pin = torch.empty(flat_netpin.numel(), dtype=torch.int32, device=dev)
        self.lane_of_pin[pin[real]] = torch.arange(self.num_slots, device=dev, dtype=torch.int32)[real]


class WeightedAverageWirelengthLanesFunction(Function):
    """WA merged forward / backward over a lane plan (dp_wa_pins_forward /
    dp_wa_pins_backward)."""

    @staticmethod
    def forward(ctx, pos, lanes, net_weights, net_mask, pin_mask, inv_gamma):
        require_cuda(pos, "pos")
        wl64 = torch.empty(REDUCE_DOUBLES, dtype=torch.float64, device=pos.device)
        grad_lane = torch.empty(2 * lanes.num_slots, dtype=torch.float32, device=pos.device)
        ig = inv_gamma.reshape(1).to(torch.float32)
        C.wa_pins_forward(pos.view(pos.numel()), lanes.group_deg, lanes.group_base, lanes.group_net, lanes.ln_pin,
                          net_weights, net_mask, ig, wl64, grad_lane)
        ctx.lanes = lanes
        ctx.grad_lane = grad_lane
        ctx.pin_mask = pin_mask
        return wl64[0].to(pos.dtype)

    @staticmethod
    def backward(ctx, grad_pos):
        g = grad_pos.reshape(1).to(torch.float32)
        mask = ctx.pin_mask.view(torch.uint8) if ctx.pin_mask is not None else None
        output = C.wa_pins_backward(ctx.grad_lane, ctx.lanes.lane_of_pin, mask, g)
        return output, None, None, None, None, None


class WeightedAverageWirelengthMergedFunction(Function):
    @staticmethod
    def forward(ctx, pos, flat_netpin, netpin_start, pin2net_map, net_weights, net_mask, pin_mask, inv_gamma):
        require_cuda(pos, "pos")
        wl, grad_intermediate = C.wa_merged_forward(pos.view(pos.numel()), flat_netpin, netpin_start, pin2net_map,
                                                    net_weights, net_mask, inv_gamma)
        ctx.pin2net_map = pin2net_map
        ctx.flat_netpin = flat_netpin
        ctx.netpin_start = netpin_start
        ctx.net_weights = net_weights
        ctx.net_mask = net_mask
        ctx.pin_mask = pin_mask
        ctx.inv_gamma = inv_gamma
        ctx.grad_intermediate = grad_intermediate
        ctx.pos = pos
        return wl

    @staticmethod
    def backward(ctx, grad_pos):
        g = grad_pos.reshape(1).to(torch.float32)
        output = C.wa_merged_backward(g, ctx.pos, ctx.grad_intermediate, ctx.flat_netpin, ctx.netpin_start,
                                      ctx.pin2net_map, ctx.net_weights, ctx.net_mask, ctx.inv_gamma, ctx.pin_mask)
        return output, None, None, None, None, None, None, None


WeightedAverageWirelengthFunction = WeightedAverageWirelengthMergedFunction
WeightedAverageWirelengthAtomicFunction = WeightedAverageWirelengthMergedFunction


class WeightedAverageWirelength(nn.Module):
    def __init__(self, flat_netpin=None, netpin_start=None, pin2net_map=None, net_weights=None, net_mask=None,
                 pin_mask=None, gamma=None, algorithm='atomic'):
        super().__init__()
        assert net_weights is not None and net_mask is not None and pin_mask is not None and gamma is not None, \
            "net_weights, net_mask, pin_mask, gamma are requried parameters"
        if algorithm not in ('net-by-net', 'atomic', 'merged'):
            raise ValueError("unknown algorithm %s" % algorithm)
        assert flat_netpin is not None and netpin_start is not None and pin2net_map is not None, \
            "flat_netpin, netpin_start, pin2net_map are requried parameters"
        self.flat_netpin = flat_netpin
        self.netpin_start = netpin_start
        self.pin2net_map = pin2net_map
        self.net_weights = net_weights
        self.net_mask = net_mask
        self.pin_mask = pin_mask
        self.gamma = gamma
        self.algorithm = algorithm
        self.lanes = None  # planned on the first call

    def forward(self, pos):
        if self.lanes is None:
            require_cuda(pos, "pos")
            self.lanes = PinLanes(self.flat_netpin, self.netpin_start)
        return WeightedAverageWirelengthLanesFunction.apply(pos, self.lanes, self.net_weights, self.net_mask,
                                                            self.pin_mask, 1.0 / self.gamma)
