"""The drop-in modules on the fast kernels.

* ``WeightedAverageWirelength`` runs the lane-per-net kernel on pin positions
  (dp_wa_pins_forward / dp_wa_pins_backward): checked against the reference's
  merged op (golden fixture of edge-case nets: degree 1, partial lane groups of
  degrees 2..8, warp nets up to 300 pins, coincident pins, exp underflow,
  masked and weighted nets) with the edge-case bar, with a pin mask, and after
  gamma changes in place between calls (the placer updates it in place).
* ``ElectricPotential`` / ``ElectricOverflow`` run the order-driven scatter and
  field gather over a visiting order (CellOrder, refreshed by the counting
  sort dp_order_cells_by_bin): checked against the reference-shaped Functions
  (per-cell kernels, themselves pinned to the reference ops) -- map, energy and
  gradient bit for bit in deterministic mode, across order refreshes and with
  the order gone stale; within the atomic-order tolerance in fp32.
"""
import math

import numpy as np
import pytest
import torch

from dreamplace_b200 import synthetic
from golden_cases import wa_cancellation_scale

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_wa_module_lane_path_edge_nets(cuda, golden):
    from dreamplace_b200.weighted_average_wirelength import (WeightedAverageWirelength,
                                                             WeightedAverageWirelengthMergedFunction)
    g = golden("wa_edge.npz")
    P = len(g["pin_pos"]) // 2
    flat, start, p2n = dev(g["flat_netpin"]), dev(g["netpin_start"]), dev(g["pin2net"])
    w, mask = dev(g["net_weights"]), dev(g["net_mask"])
    gamma = torch.tensor(float(g["gamma"]), device=cuda)
    no_mask = torch.zeros(P, dtype=torch.bool, device=cuda)
    wa = WeightedAverageWirelength(flat, start, p2n, w, mask, no_mask, gamma, algorithm="merged")
    pin = dev(g["pin_pos"]).requires_grad_(True)
    wl = wa(pin)
    wl.backward()
    assert wa.lanes is not None and int(wa.lanes.group_deg.max()) == 300
    assert math.isclose(float(wl.item()), float(g["wl"]), rel_tol=1e-5)
    ig = float(np.float32(1.0) / g["gamma"])
    scale = wa_cancellation_scale(g["pin_pos"], g["flat_netpin"], g["netpin_start"], g["net_mask"], ig)
    w_pin2 = np.tile(g["net_weights"][g["pin2net"]], 2)
    got = pin.grad.cpu().numpy()
    bar = 1e-6 + 1e-5 * np.abs(g["grad"]) + 4e-6 * scale * w_pin2
    assert np.all(np.abs(got - g["grad"]) <= bar), float(np.max(np.abs(got - g["grad"]) - bar))
    # a pin mask zeroes those pins' gradient; grad_out scales the rest
    pmask = torch.from_numpy(np.random.RandomState(3).rand(P) < 0.3).cuda()
    wa2 = WeightedAverageWirelength(flat, start, p2n, w, mask, pmask, gamma, algorithm="merged")
    pin2 = dev(g["pin_pos"]).requires_grad_(True)
    (2.5 * wa2(pin2)).backward()
    exp = 2.5 * pin.grad
    exp[torch.cat([pmask, pmask])] = 0.0
    assert torch.allclose(pin2.grad, exp, rtol=1e-6, atol=0)
    # gamma updated in place: the next call uses it, as the merged Function does
    gamma.fill_(3.0)
    pin3 = dev(g["pin_pos"]).requires_grad_(True)
    wl3 = wa(pin3)
    wl3.backward()
    pin4 = dev(g["pin_pos"]).requires_grad_(True)
    wl4 = WeightedAverageWirelengthMergedFunction.apply(pin4, flat, start, p2n, w, mask, no_mask, 1.0 / gamma)
    wl4.backward()
    assert math.isclose(float(wl3.item()), float(wl4.item()), rel_tol=1e-5)
    scale3 = wa_cancellation_scale(g["pin_pos"], g["flat_netpin"], g["netpin_start"], g["net_mask"],
                                   float(np.float32(1.0) / np.float32(3.0)))
    ref4 = pin4.grad.cpu().numpy()
    bar = 1e-6 + 1e-5 * np.abs(ref4) + 4e-6 * scale3 * w_pin2
    assert np.all(np.abs(pin3.grad.cpu().numpy() - ref4) <= bar)


def _ep(d, det, precision="fp32", fast_mode=False):
    from dreamplace_b200.electric_potential import ElectricPotential
    m = d.num_movable_nodes
    sorted_map = dev(np.argsort(d.node_size_x[:m], kind="stable").astype(np.int32))
    return ElectricPotential(dev(d.node_size_x), dev(d.node_size_y), dev(d.bin_centers(d.xl, d.xh, d.bin_size_x)),
                             dev(d.bin_centers(d.yl, d.yh, d.bin_size_y)), d.target_density, d.xl, d.yl, d.xh, d.yh,
                             d.bin_size_x, d.bin_size_y, m, d.num_terminals, d.num_filler_nodes, 0, det, sorted_map,
                             fast_mode=fast_mode, precision=precision)


def _reference_shaped(op, pos):
    """Energy and gradient through ElectricPotentialFunction (per-cell kernels)."""
    from dreamplace_b200.electric_potential import ElectricPotentialFunction
    p = pos.detach().clone().requires_grad_(True)
    e = ElectricPotentialFunction.apply(
        p, op.node_size_x_clamped, op.node_size_y_clamped, op.offset_x, op.offset_y, op.ratio, op.bin_center_x,
        op.bin_center_y, op.initial_density_map, op.target_density, op.xl, op.yl, op.xh, op.yh, op.bin_size_x,
        op.bin_size_y, op.num_movable_nodes, op.num_filler_nodes, op.padding, op.padding_mask, op.num_bins_x,
        op.num_bins_y, op.num_movable_impacted_bins_x, op.num_movable_impacted_bins_y,
        op.num_filler_impacted_bins_x, op.num_filler_impacted_bins_y, op.deterministic_flag, op.sorted_node_map,
        None, None, None, None, None, None, None, None, None, op.fast_mode, op.precision, False)
    e.backward()
    return e.detach(), p.grad.detach()


def _layouts(d):
    n, m = d.num_nodes, d.num_movable_nodes
    rng = np.random.RandomState(8)
    spread = d.initial_positions()
    spread[:m] = rng.uniform(d.xl, d.xh - 40, size=m)
    spread[n:n + m] = rng.uniform(d.yl, d.yh - 12, size=m)
    clustered = d.initial_positions()  # every movable cell near the die centre
    return {"spread": spread.astype(np.float32), "clustered": clustered.astype(np.float32)}


@pytest.mark.parametrize("layout", ["spread", "clustered"])
def test_ep_module_ordered_path_matches_per_cell_path(cuda, layout):
    d = synthetic.scaled(20000, num_bins=128, seed=9)
    pos_np = _layouts(d)[layout]
    for det in (1, 0):
        op = _ep(d, det)
        pos = dev(pos_np).requires_grad_(True)
        e = op(pos)
        e.backward()
        e_ref, g_ref = _reference_shaped(op, pos)
        if det:
            assert torch.equal(e.detach().reshape(-1), e_ref.reshape(-1))
            assert torch.equal(pos.grad, g_ref)
        else:
            assert math.isclose(float(e.item()), float(e_ref.item()), rel_tol=1e-4)
            tol = 1e-4 * float(g_ref.abs().max())
            torch.testing.assert_close(pos.grad, g_ref, rtol=1e-4, atol=tol)
        # overflow through the module (movable-only ordered scatter)
        ovf, mx = op(pos.detach(), mode="overflow")
        dm = op._density_map(pos.detach(), 0)
        from dreamplace_b200._native import C
        exp = C.density_overflow(dm, float(op.target_density * op.bin_size_x * op.bin_size_y),
                                 float(op.bin_size_x * op.bin_size_y))
        if det:
            assert float(ovf) == float(exp[0].float()) and float(mx) == float(exp[1].float())
        else:
            assert math.isclose(float(ovf), float(exp[0]), rel_tol=1e-4)


def test_ep_module_order_refresh_and_stale_order(cuda):
    """The visiting order is refreshed every `interval` calls; between
    refreshes the cells move and the order goes stale.  Deterministic results
    do not depend on either."""
    d = synthetic.scaled(20000, num_bins=128, seed=9)
    pos_np = _layouts(d)["spread"]
    op = _ep(d, 1)
    rng = np.random.RandomState(4)
    for step in range(5):
        order = op.cell_order(d.num_filler_nodes)
        order.interval = 3
        pos = dev(pos_np).requires_grad_(True)
        e = op(pos)
        e.backward()
        e_ref, g_ref = _reference_shaped(op, pos)
        assert torch.equal(e.detach().reshape(-1), e_ref.reshape(-1)), step
        assert torch.equal(pos.grad, g_ref), step
        # move the cells by up to two bins between calls
        pos_np = pos_np + rng.uniform(-2, 2, size=pos_np.shape).astype(np.float32) * np.float32(d.bin_size_x)
        pos_np[: d.num_nodes] = np.clip(pos_np[: d.num_nodes], d.xl, d.xh - 40)
        pos_np[d.num_nodes:] = np.clip(pos_np[d.num_nodes:], d.yl, d.yh - 12)
    # the order is a permutation of the scattered cells (movable, then fillers)
    o = op.cell_order(d.num_filler_nodes).order.cpu().numpy()
    m, nf, n = d.num_movable_nodes, d.num_filler_nodes, d.num_nodes
    assert np.array_equal(np.sort(o[:m]), np.arange(m))
    assert np.array_equal(np.sort(o[m:]), np.arange(n - nf, n))
