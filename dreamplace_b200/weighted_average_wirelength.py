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
"""
import torch
from torch import nn
from torch.autograd import Function

from ._native import C, require_cuda


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

    def forward(self, pos):
        return WeightedAverageWirelengthMergedFunction.apply(pos, self.flat_netpin, self.netpin_start,
                                                             self.pin2net_map, self.net_weights, self.net_mask,
                                                             self.pin_mask, 1.0 / self.gamma)
