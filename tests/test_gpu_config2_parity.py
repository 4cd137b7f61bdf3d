"""Parity at full scale: one GP trial's pieces on the 2.1M-cell design
(2.1M movable cells, 1,000 macros, 988,805 fillers, 2.2M nets, 7.09M pins,
1024 x 1024 bins) against the reference's own CPU ops (oracle/_ref), deterministic mode.

The pieces are the graph engine's own (the kernels the GP loop and the
benchmark run), called on a position set from outside:

* the density scatter of the trial (movable-only map for the overflow, and the
  movable + filler map for the Poisson solve) against
  ``electric_potential_cpp.density_map`` (reference
  ops/electric_potential/src/electric_density_map.cpp:100-152): bit-exact, and
  the fp64 overflow against the reference map's;
* the fixed-macro initial map against ``fixed_density_map``: bit-exact;
* the field gather against ``electric_force``
  (ops/electric_potential/src/electric_force.cpp:76-172) on the same field
  maps: bit-exact per node;
* the WA forward with the pin gather fused in, against ``pin_pos_cpp`` +
  ``weighted_average_wirelength_cpp_merged``
  (ops/weighted_average_wirelength/src/weighted_average_wirelength_merged.cpp:31-231):
  value within 1e-5 and every per-pin gradient within 1e-5 relative plus
  4e-6 of the two cancelling terms it is the difference of (the edge-case
  netlist's bar); the HPWL against ``hpwl_cpp`` within 1e-6.

Two layouts: the GP's initial one (every movable cell within a few units of
the die centre: one bin takes 2.1M cells, the scatter's global-atomic and
unsorted paths) and a mid-GP one (half the cells in dense clusters, half
spread)."""
import math
import os

import numpy as np
import pytest
import torch

import oracle
from dreamplace_b200 import synthetic
from golden_cases import wa_cancellation_scale
from dreamplace_b200.nonlinear_place import NonLinearPlace
from dreamplace_b200.params import Params

pytestmark = pytest.mark.gpu


def need(name):
    m = oracle.load_ref(name)
    if m is None:
        pytest.skip("reference CPU op %s not built (python oracle/build_ref.py)" % name)
    return m


@pytest.fixture(scope="module")
def setup():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.set_num_threads(os.cpu_count() or 8)
    d = synthetic.cells_2m()
    p = Params(target_density=d.target_density, stop_overflow=0.07, dct_precision="fp32", deterministic_flag=1,
               gp_noise_ratio=0.0)
    placer = NonLinearPlace(p, d)
    placer(p, d, max_iterations=2)  # builds the engine (records, lane plan, graphs)
    return d, placer.stepper.eng


def layout(d, kind):
    pos = d.initial_positions()
    if kind == "initial":
        return pos
    n, m = d.num_nodes, d.num_movable_nodes
    rng = np.random.RandomState(21)
    half = m // 2
    pos[:half] = rng.uniform(d.xl, d.xh - 40, size=half)
    pos[n:n + half] = rng.uniform(d.yl, d.yh - 12, size=half)
    centres = rng.uniform(0.1, 0.9, size=(16, 2)) * np.array([d.width, d.height])
    which = rng.randint(0, 16, size=m - half)
    sd = 0.01 * d.width
    pos[half:m] = centres[which, 0] + rng.normal(0, sd, size=m - half)
    pos[n + half:n + m] = centres[which, 1] + rng.normal(0, sd, size=m - half)
    return pos.astype(np.float32)


def t(a, dtype=None):
    x = torch.from_numpy(np.ascontiguousarray(a))
    return x if dtype is None else x.to(dtype)


@pytest.mark.parametrize("kind", ["initial", "mixed"])
def test_trial_pieces_match_reference_ops_at_2m_cells(setup, kind):
    ep_ref = need("electric_potential_cpp")
    wa_ref = need("weighted_average_wirelength_cpp_merged")
    pp_ref = need("pin_pos_cpp")
    hp_ref = need("hpwl_cpp")
    d, eng = setup
    n, m, nf, P = d.num_nodes, d.num_movable_nodes, d.num_filler_nodes, d.num_pins
    M, N = d.num_bins_x, d.num_bins_y
    bsx, bsy = d.bin_size_x, d.bin_size_y
    eng.set_position(torch.from_numpy(layout(d, kind)).cuda())
    v = eng.V[eng.slot]
    eng.refresh_order(v)
    pos = v.cpu()
    ep = eng.ep

    # stretched sizes and the fixed-macro map, as the reference module forms them
    sx, sy = t(d.node_size_x), t(d.node_size_y)
    sxc = sx.clamp(min=bsx * math.sqrt(2))
    syc = sy.clamp(min=bsy * math.sqrt(2))
    ox, oy = (sx - sxc).mul(0.5), (sy - syc).mul(0.5)
    ratio = sx * sy / (sxc * syc)
    for a, b in ((sxc, ep.node_size_x_clamped), (syc, ep.node_size_y_clamped), (ox, ep.offset_x),
                 (oy, ep.offset_y), (ratio, ep.ratio)):
        assert torch.equal(a, b.cpu())
    bcx, bcy = t(d.bin_centers(d.xl, d.xh, bsx)), t(d.bin_centers(d.yl, d.yh, bsy))
    fixed = ep_ref.fixed_density_map(pos, sx, sy, bcx, bcy, d.xl, d.yl, d.xh, d.yh, bsx, bsy, m, d.num_terminals,
                                     M, N, 0, 0, 1)
    init = fixed.mul(d.target_density)
    assert torch.equal(init.view(-1), ep.initial_density_map.view(-1).cpu())

    # density scatter: movable-only and movable + filler maps, overflow
    ovf = torch.zeros(1280, dtype=torch.float64, device="cuda")
    eng.scatter_maps(v, ovf)
    torch.cuda.synchronize()
    ref_all = ep_ref.density_map(pos, sxc, syc, ox, oy, ratio, bcx, bcy, init, d.target_density, d.xl, d.yl, d.xh,
                                 d.yh, bsx, bsy, m, nf, 0, M, N, 0, 0, 0, 0, 1)
    ref_mov = ep_ref.density_map(pos, sxc, syc, ox, oy, ratio, bcx, bcy, init, d.target_density, d.xl, d.yl, d.xh,
                                 d.yh, bsx, bsy, m, 0, 0, M, N, 0, 0, 0, 0, 1)
    assert torch.equal(eng.dmap.view(-1).cpu(), ref_all.view(-1))
    assert torch.equal(eng.omap.view(-1).cpu(), ref_mov.view(-1))
    area = bsx * bsy
    om = ref_mov.double().view(-1)
    exp_ovf = float((om - eng.ovf_target).clamp(min=0).sum())
    assert math.isclose(float(ovf[0]), exp_ovf, rel_tol=1e-9), (float(ovf[0]), exp_ovf)
    assert math.isclose(float(ovf[1]), float(om.max()) / area, rel_tol=1e-12)

    # field gather on the same field maps (seeded, of the Poisson field's scale)
    rng = np.random.RandomState(31)
    ex = t(rng.standard_normal(M * N).astype(np.float32) * 0.05)
    ey = t(rng.standard_normal(M * N).astype(np.float32) * 0.05)
    eng.grad_scale.fill_(1.0)
    eng.field_force(v, ex.cuda().view(M, N), ey.cuda().view(M, N))
    fo = eng.force_o.cpu().numpy().reshape(-1, 2)
    ref_f = ep_ref.electric_force(torch.ones(1), M, N, 0, 0, 0, 0, ex, ey, pos, sxc, syc, ox, oy, ratio, bcx, bcy,
                                  d.xl, d.yl, d.xh, d.yh, bsx, bsy, m, nf).numpy()
    order = eng.order.cpu().numpy()
    assert np.array_equal(fo[:, 0], -ref_f[order])
    assert np.array_equal(fo[:, 1], -ref_f[n + order])

    # WA forward (pin gather fused) and HPWL of the same pins
    dc = eng.data
    gamma = 0.5 * 4.0 * (bsx + bsy)
    inv_gamma = torch.tensor([1.0 / gamma], dtype=torch.float32)
    hp = torch.zeros(1280, dtype=torch.float64, device="cuda")
    eng.wirelength(v, hp, inv_gamma.cuda())
    torch.cuda.synchronize()
    pin = pp_ref.forward(pos, t(d.pin_offset_x), t(d.pin_offset_y), t(d.pin2node_map.astype(np.int64)),
                         t(d.flat_node2pin_map), t(d.flat_node2pin_start_map))
    wl, gi = wa_ref.forward(pin, t(d.flat_net2pin_map), t(d.flat_net2pin_start_map), t(d.pin2net_map),
                            t(d.net_weights), dc.net_mask_ignore_large_degrees.cpu(), inv_gamma)
    assert math.isclose(float(eng.wl64[0]), float(wl.item()), rel_tol=1e-5), (float(eng.wl64[0]), float(wl.item()))
    slot_of_pin = np.empty(P, np.int64)
    slot_of_pin[d.flat_net2pin_map] = np.arange(P)
    csr = eng.csr_pos.cpu().numpy()[slot_of_pin]
    lane = eng.lane_of_csr.cpu().numpy()[csr]
    got = eng.gnode.cpu().numpy().reshape(-1, 2)[lane]
    gi = gi.numpy()
    exp = np.stack([gi[:P], gi[P:]], axis=1)
    net_mask = dc.net_mask_ignore_large_degrees.cpu().numpy()
    mask = net_mask[d.pin2net_map].astype(bool)
    # the WA gradient of a pin is a difference of two terms of size ~|x| / gamma
    # times the gradient's own scale (x / gamma ~ 100 on this die); CUDA's and
    # glibc's expf differ by an ulp here and there, which moves such a gradient
    # by a few 1e-7 of those terms (wa_cancellation_scale): the bar is the one
    # the edge-case netlist test uses
    scale = wa_cancellation_scale(pin.numpy(), d.flat_net2pin_map, d.flat_net2pin_start_map, net_mask,
                                  float(inv_gamma.item()))
    scale = np.stack([scale[:P], scale[P:]], axis=1)
    bar = 1e-6 + 1e-5 * np.abs(exp) + 4e-6 * scale
    err = np.abs(got - exp)
    assert np.all(err[mask] <= bar[mask]), float(np.max(err[mask] - bar[mask]))
    print(kind, "WA gradient: max |err| / bar %.3f, max |err| %.3e, pins beyond 1e-5 relative: %d of %d"
          % (float(np.max(err[mask] / bar[mask])), float(err[mask].max()),
             int(np.sum(err[mask] > 1e-5 * np.abs(exp[mask]) + 1e-6)), int(mask.sum()) * 2))
    ref_hp = float(hp_ref.forward(pin, t(d.flat_net2pin_map), t(d.flat_net2pin_start_map), t(d.net_weights),
                                  dc.net_mask_all.cpu()).item())
    assert math.isclose(float(hp[0]), ref_hp, rel_tol=1e-6), (float(hp[0]), ref_hp)
