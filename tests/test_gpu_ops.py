"""GPU parity of every hot-path kernel against the CPU oracle and the reference's
own CPU ops (golden fixtures).  Bars: bit-exact for fixed-point maps, the
deterministic force and all pin/net indexing; <= 1e-5 relative for fp32
gradients; the stated tolerance per Poisson-solve precision."""
import math

import numpy as np
import pytest
import torch

import oracle
from dreamplace_b200 import synthetic
from golden_cases import ep_unit_case, wa_cancellation_scale, wa_edge_netlist, window_to_map

pytestmark = pytest.mark.gpu

# Poisson-solve error bars against the fp64 oracle, relative to the max |value|
FIELD_TOL = {"fp32": 2e-5, "tf32": 5e-3, "bf16": 3e-2, "split_bf16": 2e-4}


@pytest.fixture(scope="module")
def C():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dreamplace_b200._native import C
    return C


def dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return t if dtype is None else t.to(dtype)


def small_design():
    return synthetic.scaled(3000, num_bins=64, seed=7, name="golden_small")


def stretched_t(d):
    sx, sy = dev(d.node_size_x), dev(d.node_size_y)
    sxc = sx.clamp(min=d.bin_size_x * math.sqrt(2))
    syc = sy.clamp(min=d.bin_size_y * math.sqrt(2))
    return sx, sy, sxc, syc, (sx - sxc).mul(0.5), (sy - syc).mul(0.5), sx * sy / (sxc * syc)


def sorted_map(d):
    return dev(np.argsort(d.node_size_x[:d.num_movable_nodes], kind="stable").astype(np.int32))


def test_fixed_density_map(C, golden):
    g = golden("design_small.npz")
    d = small_design()
    pos = dev(g["pos"])
    sx, sy = dev(d.node_size_x), dev(d.node_size_y)
    bcx = dev(d.bin_centers(d.xl, d.xh, d.bin_size_x))
    bcy = dev(d.bin_centers(d.yl, d.yh, d.bin_size_y))
    for det in (0, 1):
        out = C.fixed_density_map(pos, sx, sy, bcx, bcy, d.xl, d.yl, d.xh, d.yh, d.bin_size_x, d.bin_size_y,
                                  d.num_movable_nodes, d.num_terminals, d.num_bins_x, d.num_bins_y, 0, 0, det)
        ref = g["fixed_map_det%d" % det].reshape(-1)
        got = out.cpu().numpy().reshape(-1)
        if det:
            assert np.array_equal(got, ref)
        else:
            np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-3)


@pytest.mark.parametrize("sorted_nodes", [False, True])
def test_density_map_deterministic_bit_exact(C, golden, sorted_nodes):
    g = golden("design_small.npz")
    d = small_design()
    pos = dev(g["pos"])
    sx, sy, sxc, syc, ox, oy, ratio = stretched_t(d)
    init = dev(g["fixed_map_det1"]).mul(d.target_density).view(-1)
    snm = sorted_map(d) if sorted_nodes else None
    out = C.density_map(pos, sxc, syc, ox, oy, ratio, init, init, init, d.target_density, d.xl, d.yl, d.xh, d.yh,
                        d.bin_size_x, d.bin_size_y, d.num_movable_nodes, d.num_filler_nodes, 0, d.num_bins_x,
                        d.num_bins_y, 0, 0, 0, 0, 1, snm)
    assert np.array_equal(out.cpu().numpy().reshape(-1), g["density_map_det1"].reshape(-1))
    # the integer map itself against the C oracle's
    fx = C.density_map_fixed_point(pos, sxc, syc, ox, oy, ratio, d.xl, d.yl, d.xh, d.yh, d.bin_size_x,
                                   d.bin_size_y, d.num_movable_nodes, d.num_filler_nodes, d.num_bins_x,
                                   d.num_bins_y, snm)
    s = oracle.stretched(d.node_size_x, d.node_size_y, d.bin_size_x, d.bin_size_y)
    _, ofx = oracle.triangle_density_map(g["pos"], *s, d.num_nodes, d.num_movable_nodes, d.num_filler_nodes,
                                         d.num_bins_x, d.num_bins_y, d.xl, d.yl, d.xh, d.yh, d.bin_size_x,
                                         d.bin_size_y, deterministic=True)
    assert np.array_equal(fx.cpu().numpy(), ofx)


def test_density_map_fp32(C, golden):
    g = golden("design_small.npz")
    d = small_design()
    pos = dev(g["pos"])
    sx, sy, sxc, syc, ox, oy, ratio = stretched_t(d)
    init = dev(g["fixed_map_det0"]).mul(d.target_density).view(-1)
    out = C.density_map(pos, sxc, syc, ox, oy, ratio, init, init, init, d.target_density, d.xl, d.yl, d.xh, d.yh,
                        d.bin_size_x, d.bin_size_y, d.num_movable_nodes, d.num_filler_nodes, 0, d.num_bins_x,
                        d.num_bins_y, 0, 0, 0, 0, 0, sorted_map(d))
    ref = g["density_map_det0"].reshape(-1)
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-5, atol=1e-5 * float(np.max(np.abs(ref))))


def test_density_map_clustered_start(C):
    """All movable cells at the die centre (GP iteration 0): the warp-combined
    atomics must still produce the oracle's integer map exactly."""
    d = synthetic.cells_10k()
    pos = d.initial_positions()
    sx, sy, sxc, syc, ox, oy, ratio = stretched_t(d)
    fx = C.density_map_fixed_point(dev(pos), sxc, syc, ox, oy, ratio, d.xl, d.yl, d.xh, d.yh, d.bin_size_x,
                                   d.bin_size_y, d.num_movable_nodes, d.num_filler_nodes, d.num_bins_x,
                                   d.num_bins_y, sorted_map(d))
    s = oracle.stretched(d.node_size_x, d.node_size_y, d.bin_size_x, d.bin_size_y)
    _, ofx = oracle.triangle_density_map(pos, *s, d.num_nodes, d.num_movable_nodes, d.num_filler_nodes,
                                         d.num_bins_x, d.num_bins_y, d.xl, d.yl, d.xh, d.yh, d.bin_size_x,
                                         d.bin_size_y, deterministic=True)
    assert np.array_equal(fx.cpu().numpy(), ofx)


def test_electric_force_bit_exact(C, golden):
    g = golden("design_small.npz")
    d = small_design()
    pos = dev(g["pos"])
    sx, sy, sxc, syc, ox, oy, ratio = stretched_t(d)
    grad = torch.ones(1, device="cuda")
    for snm in (None, sorted_map(d)):
        out = C.electric_force(grad, d.num_bins_x, d.num_bins_y, 0, 0, 0, 0, dev(g["field_x"]).view(-1),
                               dev(g["field_y"]).view(-1), pos, sxc, syc, ox, oy, ratio, pos, pos, d.xl, d.yl, d.xh,
                               d.yh, d.bin_size_x, d.bin_size_y, d.num_movable_nodes, d.num_filler_nodes, 1, snm,
                               -1.0)
        assert np.array_equal(out.cpu().numpy(), g["force"])


def test_pin_pos_and_hpwl(C, golden):
    g = golden("design_small.npz")
    d = small_design()
    pos = dev(g["pos"])
    pin = C.pin_pos_forward(pos, dev(d.pin_offset_x), dev(d.pin_offset_y), dev(d.pin2node_map))
    assert np.array_equal(pin.cpu().numpy(), g["pin_pos"])
    back = C.pin_pos_backward(dev(g["pin_grad_in"]), pos, dev(d.flat_node2pin_map), dev(d.flat_node2pin_start_map),
                              d.num_physical_nodes)
    assert np.array_equal(back.cpu().numpy(), g["pin_pos_backward"])
    deg = np.diff(d.flat_net2pin_start_map)
    h = C.hpwl_forward(pin, dev(d.flat_net2pin_map), dev(d.flat_net2pin_start_map), dev(d.net_weights),
                       dev((deg >= 2).astype(np.uint8)))
    ho = oracle.hpwl(g["pin_pos"], d.flat_net2pin_map, d.flat_net2pin_start_map, (deg >= 2).astype(np.uint8),
                     d.net_weights)
    assert math.isclose(float(h.item()), ho, rel_tol=1e-12)
    assert math.isclose(float(h.item()), float(g["hpwl"]), rel_tol=1e-5)


def test_wa_merged_forward_backward(C, golden):
    g = golden("design_small.npz")
    d = small_design()
    pin = dev(g["pin_pos"])
    mask = dev(g["net_mask"])
    inv_gamma = torch.tensor([float(g["inv_gamma"])], device="cuda")
    wl, gi = C.wa_merged_forward(pin, dev(d.flat_net2pin_map), dev(d.flat_net2pin_start_map), dev(d.pin2net_map),
                                 dev(d.net_weights), mask, inv_gamma)
    assert math.isclose(float(wl.item()), float(g["wa_wl"]), rel_tol=1e-5)
    np.testing.assert_allclose(gi.cpu().numpy(), g["wa_grad_intermediate"], rtol=1e-5, atol=1e-6)
    pin_mask = dev((d.pin2node_map >= d.num_movable_nodes).astype(np.uint8))
    grad = torch.full((1,), 0.5, device="cuda")
    out = C.wa_merged_backward(grad, pin, gi.clone(), dev(d.flat_net2pin_map), dev(d.flat_net2pin_start_map),
                               dev(d.pin2net_map), dev(d.net_weights), mask, inv_gamma, pin_mask)
    exp = g["wa_grad_intermediate"] * np.float32(0.5)
    pm = np.concatenate([d.pin2node_map >= d.num_movable_nodes] * 2)
    exp[pm] = 0
    np.testing.assert_allclose(out.cpu().numpy(), exp, rtol=1e-5, atol=1e-6)


def test_wa_unit_golden(C, golden):
    g = golden("wa_unit.npz")
    inv_gamma = torch.tensor([1.0 / float(g["gamma"])], device="cuda")
    wl, gi = C.wa_merged_forward(dev(g["pos"]), dev(g["flat_netpin"]), dev(g["netpin_start"]), dev(g["pin2net"]),
                                 dev(g["net_weights"]), dev(g["net_mask"]), inv_gamma)
    assert math.isclose(float(wl.item()), float(g["wl"]), rel_tol=1e-6)
    out = C.wa_merged_backward(torch.ones(1, device="cuda"), dev(g["pos"]), gi, dev(g["flat_netpin"]),
                               dev(g["netpin_start"]), dev(g["pin2net"]), dev(g["net_weights"]), dev(g["net_mask"]),
                               inv_gamma, None)
    np.testing.assert_allclose(out.cpu().numpy(), g["grad"], rtol=1e-6, atol=1e-7)


def test_ops_unit_cases(C, golden):
    """The reference's own unit-test cases of hpwl, pin_pos and move_boundary
    (unittest/ops/{hpwl,pin_pos,move_boundary}_unittest.py) through the CUDA
    ops: pin_pos forward / backward and move_boundary bit for bit against the
    reference's CPU ops, the HPWL to the float32 total they return."""
    g = golden("ops_unit.npz")
    h = C.hpwl_forward(dev(g["hpwl_pin_pos"]), dev(g["hpwl_flat_netpin"]), dev(g["hpwl_netpin_start"]),
                       dev(g["hpwl_net_weights"]), dev(g["hpwl_net_mask"]))
    assert math.isclose(float(h.item()), float(g["hpwl"]), rel_tol=1e-6)
    pos = dev(g["pp_pos"])
    pin = C.pin_pos_forward(pos, dev(g["pp_offset_x"]), dev(g["pp_offset_y"]), dev(g["pp_pin2node"]))
    assert np.array_equal(pin.cpu().numpy(), g["pin_pos"])
    back = C.pin_pos_backward(torch.ones(2 * len(g["pp_pin2node"]), device="cuda"), pos, dev(g["pp_flat_node2pin"]),
                              dev(g["pp_node_start"]), int(g["pp_num_physical"]))
    assert np.array_equal(back.cpu().numpy(), g["pin_pos_backward"])
    moved = dev(g["mb_pos"])
    C.move_boundary_forward(moved, dev(g["mb_node_size_x"]), dev(g["mb_node_size_y"]), *[float(v) for v in g["mb_box"]],
                            int(g["mb_num_movable"]), int(g["mb_num_filler"]))
    assert np.array_equal(moved.cpu().numpy(), g["move_boundary"])


def test_move_boundary_and_pws(C):
    d = synthetic.cells_10k()
    pos = d.initial_positions()
    pos[:100] = -50.0
    pos[d.num_nodes:d.num_nodes + 100] = 1e5
    t = dev(pos)
    C.move_boundary_forward(t, dev(d.node_size_x), dev(d.node_size_y), d.xl, d.yl, d.xh, d.yh, d.num_movable_nodes,
                            d.num_filler_nodes)
    exp = pos.copy()
    n = d.num_nodes
    idx = np.r_[0:d.num_movable_nodes, n - d.num_filler_nodes:n]
    sx, sy = d.node_size_x, d.node_size_y
    exp[idx] = np.minimum(np.maximum(pos[idx], np.float32(d.xl)), (np.float32(d.xh) - sx[idx]).astype(np.float32))
    exp[n + idx] = np.minimum(np.maximum(pos[n + idx], np.float32(d.yl)), (np.float32(d.yh) - sy[idx]).astype(np.float32))
    assert np.array_equal(t.cpu().numpy(), exp)
    w = np.random.RandomState(3).uniform(0.5, 2, size=d.num_nets).astype(np.float32)
    out = C.pws_forward(dev(w), dev(d.flat_node2pin_map), dev(d.flat_node2pin_start_map), dev(d.pin2net_map),
                        d.num_nodes).cpu().numpy()
    exp = np.zeros(d.num_nodes, np.float32)
    for i in range(d.num_physical_nodes):
        s = np.float32(0)
        for j in range(d.flat_node2pin_start_map[i], d.flat_node2pin_start_map[i + 1]):
            s = np.float32(s + w[d.pin2net_map[d.flat_node2pin_map[j]]])
        exp[i] = s
    assert np.array_equal(out, exp)


@pytest.mark.parametrize("precision", ["fp32", "tf32", "bf16", "split_bf16"])
@pytest.mark.parametrize("shape", [(64, 64), (128, 256), (1024, 1024)])
def test_transforms_against_fp64(C, precision, shape):
    from dreamplace_b200 import dct2_fft2 as dct
    M, N = shape
    x = np.random.RandomState(M + N).uniform(-1, 1, size=(M, N)).astype(np.float32)
    xt = dev(x)
    for cls, f in ((dct.DCT2, oracle.dct2), (dct.IDCT2, oracle.idct2), (dct.IDCT_IDXST, oracle.idct_idxst),
                   (dct.IDXST_IDCT, oracle.idxst_idct)):
        got = cls(precision=precision)(xt).cpu().numpy().astype(np.float64)
        ref = f(x)
        err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
        assert err <= FIELD_TOL[precision], (cls.__name__, precision, shape, err)
    assert C.tc_status() == 0


@pytest.mark.parametrize("precision", ["fp32", "tf32", "bf16", "split_bf16"])
def test_poisson_solve_against_fp64(C, golden, precision):
    from dreamplace_b200.electric_potential import poisson_solve
    g = golden("design_small.npz")
    d = small_design()
    dm = g["density_map_det1"].reshape(d.num_bins_x, d.num_bins_y)
    rho = dev(dm).mul_(1.0 / (d.bin_size_x * d.bin_size_y))
    ex, ey, energy = poisson_solve(rho, d.bin_size_x, d.bin_size_y, precision)
    rex, rey, renergy = oracle.poisson(dm, d.bin_size_x, d.bin_size_y)
    for got, ref in ((ex, rex), (ey, rey)):
        err = np.max(np.abs(got.cpu().numpy() - ref)) / np.max(np.abs(ref))
        assert err <= FIELD_TOL[precision], (precision, err)
    assert abs(float(energy.item()) - renergy) <= FIELD_TOL[precision] * abs(renergy) * 10
    assert C.tc_status() == 0


def test_electric_potential_module_fwd_bwd(C, golden):
    """Module-level drop-in: energy and gradient against the reference's FFT
    pipeline outputs (golden) in deterministic mode."""
    from dreamplace_b200.electric_potential import ElectricPotential
    g = golden("design_small.npz")
    d = small_design()
    pos = dev(g["pos"]).requires_grad_(True)
    op = ElectricPotential(dev(d.node_size_x), dev(d.node_size_y), dev(d.bin_centers(d.xl, d.xh, d.bin_size_x)),
                           dev(d.bin_centers(d.yl, d.yh, d.bin_size_y)), d.target_density, d.xl, d.yl, d.xh, d.yh,
                           d.bin_size_x, d.bin_size_y, d.num_movable_nodes, d.num_terminals, d.num_filler_nodes, 0,
                           True, sorted_map(d), precision="fp32")
    energy = op(pos)
    assert math.isclose(float(energy.item()), float(g["energy"]), rel_tol=1e-4)
    energy.backward()
    ref = g["force"]
    err = np.max(np.abs(pos.grad.cpu().numpy() - ref)) / np.max(np.abs(ref))
    assert err <= 1e-4
    ovf, mx = op(pos.detach(), mode="overflow")
    assert float(ovf) >= 0 and float(mx) > 0


def test_density_map_exact_against_reference(C):
    ref = oracle.load_ref("density_map_cpp")
    if ref is None:
        pytest.skip("reference density_map_cpp not built")
    from dreamplace_b200.placement_ops import DensityMap
    d = synthetic.cells_10k()
    pos = d.initial_positions()
    rng = np.random.RandomState(5)
    m = d.num_movable_nodes
    pos[:m] = rng.uniform(d.xl, d.xh, size=m)
    pos[d.num_nodes:d.num_nodes + m] = rng.uniform(d.yl, d.yh, size=m)
    ranges = [(0, m), (d.num_nodes - d.num_filler_nodes, d.num_nodes)]
    for det in (0, 1):
        exp = torch.zeros(d.num_bins_x, d.num_bins_y)
        for b, e in ranges:
            exp = ref.forward(torch.from_numpy(pos), torch.from_numpy(d.node_size_x), torch.from_numpy(d.node_size_y),
                              exp, d.xl, d.yl, d.xh, d.yh, d.num_bins_x, d.num_bins_y, b, e, det)
        op = DensityMap(dev(d.node_size_x), dev(d.node_size_y), d.xl, d.yl, d.xh, d.yh, d.num_bins_x, d.num_bins_y,
                        ranges, det)
        got = op.forward(dev(pos)).cpu().numpy()
        if det:
            assert np.array_equal(got, exp.numpy())
        else:
            np.testing.assert_allclose(got, exp.numpy(), rtol=1e-5, atol=1e-3)


def spatial_order(d, pos, idx):
    """The engine's visiting order: cells sorted by the bin where their
    stretched footprint starts, 16x16-bin tiles in serpentine order."""
    n = d.num_nodes
    s = oracle.stretched(d.node_size_x, d.node_size_y, d.bin_size_x, d.bin_size_y)
    ox, oy = s[2], s[3]
    kx = np.clip(((pos[idx] + ox[idx] - d.xl) / d.bin_size_x).astype(np.int64), 0, d.num_bins_x - 1)
    hy = np.clip(((pos[n + idx] + oy[idx] - d.yl) / d.bin_size_y).astype(np.int64), 0, d.num_bins_y - 1)
    ty = (d.num_bins_y + 15) >> 4
    tx, tyy = kx >> 4, hy >> 4
    tyy = np.where(tx & 1, ty - 1 - tyy, tyy)
    key = ((tx * ty + tyy) << 8) | ((kx & 15) << 4) | (hy & 15)
    return idx[np.argsort(key, kind="stable")].astype(np.int32)


def pack_xy(pos, n):
    return dev(np.stack([pos[:n], pos[n:]], axis=1).reshape(-1).astype(np.float32))


def order_xy(C, xy, order):
    """Positions in visiting order (what the trial kernel maintains)."""
    out = torch.empty(2 * len(order), device="cuda")
    C.gather_order_xy(xy, dev(order), len(order), out)
    return out


def records(C, d, order):
    sx, sy, sxc, syc, ox, oy, ratio = stretched_t(d)
    rec4 = torch.empty(4 * len(order), device="cuda")
    ratio_o = torch.empty(len(order), device="cuda")
    inv = torch.zeros(d.num_nodes, dtype=torch.int32, device="cuda")
    C.build_cell_records(sxc, syc, ox, oy, ratio, dev(order), len(order), rec4, ratio_o, inv)
    return rec4, ratio_o, inv


@pytest.mark.parametrize("layout", ["clustered", "spread"])
def test_ordered_tiled_scatter(C, layout):
    """The order-driven scatter over per-cell records (register, shared-tile and
    global paths): integer map bit-exact with the oracle for any visiting order;
    fp32 map within atomic-order tolerance."""
    d = synthetic.scaled(20000, num_bins=128, seed=9)
    pos = d.initial_positions()
    n, m = d.num_nodes, d.num_movable_nodes
    if layout == "spread":
        rng = np.random.RandomState(1)
        pos[:m] = rng.uniform(d.xl, d.xh - 40, size=m)
        pos[n:n + m] = rng.uniform(d.yl, d.yh - 12, size=m)
    s = oracle.stretched(d.node_size_x, d.node_size_y, d.bin_size_x, d.bin_size_y)
    ref_map, ref_fx = oracle.triangle_density_map(pos, *s, n, m, d.num_filler_nodes, d.num_bins_x, d.num_bins_y,
                                                  d.xl, d.yl, d.xh, d.yh, d.bin_size_x, d.bin_size_y,
                                                  deterministic=True)
    f32_map, _ = oracle.triangle_density_map(pos, *s, n, m, d.num_filler_nodes, d.num_bins_x, d.num_bins_y,
                                             d.xl, d.yl, d.xh, d.yh, d.bin_size_x, d.bin_size_y)
    idx = np.r_[0:m, n - d.num_filler_nodes:n].astype(np.int32)
    xy = pack_xy(pos, n)
    orders = (idx, np.random.RandomState(2).permutation(idx).astype(np.int32),
              np.r_[spatial_order(d, pos, idx[:m]), spatial_order(d, pos, idx[m:])].astype(np.int32))
    for order in orders:
        rec4, ratio_o, _ = records(C, d, order)
        out = torch.empty(d.num_bins_x * d.num_bins_y, device="cuda")
        scratch = torch.empty(d.num_bins_x * d.num_bins_y, dtype=torch.int64, device="cuda")
        C.density_map_ordered_into(order_xy(C, xy, order), rec4, ratio_o, len(order), None, d.xl, d.yl, d.xh, d.yh,
                                   d.bin_size_x, d.bin_size_y, d.num_bins_x, d.num_bins_y, 1, scratch, out)
        assert np.array_equal(scratch.cpu().numpy(), ref_fx)
        assert np.array_equal(out.cpu().numpy(), ref_map)
        C.density_map_ordered_into(order_xy(C, xy, order), rec4, ratio_o, len(order), None, d.xl, d.yl, d.xh, d.yh,
                                   d.bin_size_x, d.bin_size_y, d.num_bins_x, d.num_bins_y, 0, None, out)
        np.testing.assert_allclose(out.cpu().numpy(), f32_map, rtol=1e-4, atol=1e-4 * float(np.max(f32_map)))


def test_ordered_force_and_fused_assembly(C, golden):
    """Field gather over records in visiting order: bit-exact with the golden
    force per node.  Fused gradient assembly + preconditioner + step-size norms:
    the gradient bit-exact with pin sum + force + dp_precondition_step_size, the
    fp64 norms equal up to summation order."""
    g = golden("design_small.npz")
    d = small_design()
    n, m, nf = d.num_nodes, d.num_movable_nodes, d.num_filler_nodes
    pos_np = g["pos"].astype(np.float32)
    idx = np.r_[0:m, n - nf:n].astype(np.int32)
    order = np.r_[spatial_order(d, pos_np, idx[:m]), spatial_order(d, pos_np, idx[m:])].astype(np.int32)
    rec4, ratio_o, inv = records(C, d, order)
    xy = pack_xy(pos_np, n)
    grad = torch.ones(1, device="cuda")
    force_o = torch.empty(2 * len(order), device="cuda")
    fx, fy = dev(g["field_x"]).view(-1), dev(g["field_y"]).view(-1)
    C.electric_force_ordered(grad, fx, fy, order_xy(C, xy, order), rec4, ratio_o, len(order), d.xl, d.yl, d.bin_size_x,
                             d.bin_size_y, d.num_bins_x, d.num_bins_y, -1.0, force_o)
    fo = force_o.cpu().numpy().reshape(-1, 2)
    assert np.array_equal(fo[:, 0], g["force"][order])
    assert np.array_equal(fo[:, 1], g["force"][n + order])

    # wirelength pin gradient in node-CSR order: any values exercise the sum
    rng = np.random.RandomState(5)
    node_start = dev(d.flat_node2pin_start_map.astype(np.int32))
    gnode = dev(rng.standard_normal(2 * d.num_pins).astype(np.float32))
    pws = dev(rng.uniform(0, 5, n).astype(np.float32))
    area = dev((d.node_size_x * d.node_size_y).astype(np.float32))
    lam = torch.tensor([1e-3], device="cuda")
    v = dev(pos_np)
    v_new = v + dev(rng.standard_normal(2 * n).astype(np.float32))
    g_old = dev(rng.standard_normal(2 * n).astype(np.float32))
    st_ref = torch.zeros(8 + 2 * 1280, dtype=torch.float64, device="cuda")
    st_got = st_ref.clone()
    sx, sy, sxc, syc, ox, oy, ratio = stretched_t(d)
    exp = torch.empty(2 * n, device="cuda")
    C.electric_force_into(grad, fx, fy, v, sxc, syc, ox, oy, ratio, d.xl, d.yl, d.xh, d.yh, d.bin_size_x,
                          d.bin_size_y, d.num_bins_x, d.num_bins_y, m, nf, None, -1.0, exp)
    C.node_pin_sum(gnode, node_start, grad, m, 1, exp)
    C.precondition_step_size(exp, g_old, v_new, v, pws, area, lam, st_ref)
    got = torch.empty(2 * n, device="cuda")
    C.assemble_precondition_step(gnode, node_start, grad, force_o, inv, m, nf, pws, area, lam, v_new, v, g_old, got,
                                 st_got, None)
    # the same pin gradients stored in another order, gathered through grad_index
    perm = np.random.RandomState(8).permutation(d.num_pins)
    shuffled = torch.empty_like(gnode).view(-1, 2)
    shuffled[dev(perm).long()] = gnode.view(-1, 2)
    got2 = torch.empty(2 * n, device="cuda")
    st2 = torch.zeros_like(st_ref)
    C.assemble_precondition_step(shuffled.reshape(-1), node_start, grad, force_o, inv, m, nf, pws, area, lam, v_new, v,
                                 g_old, got2, st2, dev(perm.astype(np.int32)))
    assert torch.equal(got2, exp)
    assert torch.equal(got, exp)
    np.testing.assert_allclose(st_got[:8].cpu().numpy(), st_ref[:8].cpu().numpy(), rtol=1e-12)


def test_fused_assembly_long_pin_ranges(C):
    """The assembly's staged gather on node tiles whose pins overflow one
    shared-memory chunk (nodes of up to 5000 pins, ranges crossing chunk
    edges, nodes without pins, fixed nodes between movable and filler ones):
    bit-exact with the separate pin-sum and precondition kernels."""
    rng = np.random.RandomState(11)
    m, nfix, nf = 3000, 40, 700
    n = m + nfix + nf
    deg = rng.randint(0, 7, size=n)
    deg[rng.choice(m, 12, replace=False)] = rng.randint(1500, 5000, size=12)
    deg[m:m + nfix] = rng.randint(0, 20, size=nfix)
    deg[m + nfix:] = 0
    start = np.zeros(n + 1, np.int64)
    np.cumsum(deg, out=start[1:])
    P = int(start[-1])
    node_start = dev(start.astype(np.int32))
    gnode = dev(rng.standard_normal(2 * P).astype(np.float32))
    grad = torch.tensor([0.37], device="cuda")
    pws = dev(rng.uniform(0, 5, n).astype(np.float32))
    area = dev(rng.uniform(0, 400, n).astype(np.float32))
    lam = torch.tensor([1e-2], device="cuda")
    v = dev(rng.standard_normal(2 * n).astype(np.float32))
    v_new = v + dev(rng.standard_normal(2 * n).astype(np.float32))
    g_old = dev(rng.standard_normal(2 * n).astype(np.float32))
    inv = dev(rng.permutation(m + nf).astype(np.int32))
    inv_full = torch.zeros(n, dtype=torch.int32, device="cuda")
    inv_full[:m] = inv[:m]
    inv_full[m + nfix:] = inv[m:]
    force_o = dev(rng.standard_normal(2 * (m + nf)).astype(np.float32))
    fo = force_o.view(-1, 2)
    exp = torch.zeros(2 * n, device="cuda")
    mov_or_fill = torch.cat([torch.arange(m), torch.arange(m + nfix, n)]).cuda()
    exp[mov_or_fill] = fo[inv_full[mov_or_fill].long(), 0]
    exp[n + mov_or_fill] = fo[inv_full[mov_or_fill].long(), 1]
    C.node_pin_sum(gnode, node_start, grad, m, 1, exp)
    st_ref = torch.zeros(8 + 2 * 1280, dtype=torch.float64, device="cuda")
    C.precondition_step_size(exp, g_old, v_new, v, pws, area, lam, st_ref)
    st_got = torch.zeros_like(st_ref)
    got = torch.empty(2 * n, device="cuda")
    C.assemble_precondition_step(gnode, node_start, grad, force_o, inv_full, m, nf, pws, area, lam, v_new, v, g_old,
                                 got, st_got, None)
    assert torch.equal(got, exp)
    np.testing.assert_allclose(st_got[:8].cpu().numpy(), st_ref[:8].cpu().numpy(), rtol=1e-12)


def test_ordered_split_scatter(C):
    """Two maps from one pass (movable prefix, all cells): bit-exact with two
    separate fixed-point scatters; fp32 within atomic-order tolerance."""
    d = synthetic.scaled(20000, num_bins=128, seed=9)
    pos = d.initial_positions()
    n, m, nf = d.num_nodes, d.num_movable_nodes, d.num_filler_nodes
    rng = np.random.RandomState(3)
    pos[:m] = rng.normal((d.xl + d.xh) / 2, 0.05 * (d.xh - d.xl), size=m).clip(d.xl, d.xh - 40)
    pos[n:n + m] = rng.normal((d.yl + d.yh) / 2, 0.05 * (d.yh - d.yl), size=m).clip(d.yl, d.yh - 12)
    idx = np.r_[0:m, n - nf:n].astype(np.int32)
    order = np.r_[spatial_order(d, pos, idx[:m]), spatial_order(d, pos, idx[m:])].astype(np.int32)
    rec4, ratio_o, _ = records(C, d, order)
    xy = pack_xy(pos, n)
    nb = d.num_bins_x * d.num_bins_y
    init = dev(np.random.RandomState(4).uniform(0, 50, nb).astype(np.float32))
    scratch = torch.empty(nb, dtype=torch.int64, device="cuda")
    geo = (d.xl, d.yl, d.xh, d.yh, d.bin_size_x, d.bin_size_y, d.num_bins_x, d.num_bins_y)
    for det in (1, 0):
        first, full = torch.empty(nb, device="cuda"), torch.empty(nb, device="cuda")
        ovf = torch.zeros(1280, dtype=torch.float64, device="cuda")
        ba = d.bin_size_x * d.bin_size_y
        C.density_map_ordered_split(order_xy(C, xy, order), rec4, ratio_o, m, len(order), init, *geo, det,
                                    scratch if det else None, first, full, 0.9 * ba, ba, ovf)
        exp_first, exp_full = torch.empty(nb, device="cuda"), torch.empty(nb, device="cuda")
        C.density_map_ordered_into(order_xy(C, xy, order), rec4, ratio_o, m, init, *geo, det, scratch if det else None,
                                   exp_first)
        C.density_map_ordered_into(order_xy(C, xy, order), rec4, ratio_o, len(order), init, *geo, det,
                                   scratch if det else None, exp_full)
        exp_ovf = torch.zeros(1280, dtype=torch.float64, device="cuda")
        C.density_overflow_into(first, 0.9 * ba, ba, exp_ovf)
        torch.testing.assert_close(ovf[:2], exp_ovf[:2], rtol=1e-12, atol=0)
        if det:
            assert torch.equal(first, exp_first) and torch.equal(full, exp_full)
        else:
            tol = 1e-4 * float(exp_full.abs().max())
            torch.testing.assert_close(first, exp_first, rtol=1e-4, atol=tol)
            torch.testing.assert_close(full, exp_full, rtol=1e-4, atol=tol)
        # node-order positions read through the order: the same maps and overflow
        first2, full2 = torch.empty(nb, device="cuda"), torch.empty(nb, device="cuda")
        ovf2 = torch.zeros(1280, dtype=torch.float64, device="cuda")
        C.density_map_ordered_split(xy, rec4, ratio_o, m, len(order), init, *geo, det, scratch if det else None,
                                    first2, full2, 0.9 * ba, ba, ovf2, order=dev(order))
        if det:
            assert torch.equal(first2, first) and torch.equal(full2, full) and torch.equal(ovf2[:2], ovf[:2])
        else:
            tol = 1e-4 * float(full.abs().max())
            torch.testing.assert_close(full2, full, rtol=1e-4, atol=tol)
    # the field gather through the order equals the gather from the ordered copy
    fx = dev(np.random.RandomState(5).standard_normal(nb).astype(np.float32))
    fy = dev(np.random.RandomState(6).standard_normal(nb).astype(np.float32))
    grad = torch.tensor([0.5], device="cuda")
    fo1 = torch.empty(2 * len(order), device="cuda")
    fo2 = torch.empty_like(fo1)
    C.electric_force_ordered(grad, fx, fy, order_xy(C, xy, order), rec4, ratio_o, len(order), d.xl, d.yl,
                             d.bin_size_x, d.bin_size_y, d.num_bins_x, d.num_bins_y, -1.0, fo1)
    C.electric_force_ordered(grad, fx, fy, xy, rec4, ratio_o, len(order), d.xl, d.yl, d.bin_size_x, d.bin_size_y,
                             d.num_bins_x, d.num_bins_y, -1.0, fo2, order=dev(order))
    assert torch.equal(fo1, fo2)


def lane_inputs(C, d, net_order=None):
    """Slot (flat_netpin) arrays, node-CSR positions and the lane plan of a design
    (nets placed in ``net_order``, a permutation; None: index order)."""
    P = d.num_pins
    fnp = d.flat_net2pin_map.astype(np.int64)
    slot_of_pin = np.empty(P, np.int64)
    slot_of_pin[fnp] = np.arange(P)
    node_slots = slot_of_pin[d.flat_node2pin_map]
    csr_pos = np.empty(P, np.int64)
    csr_pos[node_slots] = np.arange(P)
    g_deg, g_base, g_net, l_slot = C.plan_net_lanes(torch.from_numpy(d.flat_net2pin_start_map.astype(np.int32)),
                                                    None if net_order is None else
                                                    torch.from_numpy(net_order.astype(np.int32)))
    ls = l_slot.numpy().astype(np.int64)
    real = ls >= 0
    ls = np.where(real, ls, 0)
    ln_node = np.where(real, d.pin2node_map[fnp][ls], 0).astype(np.int32)
    ln_offx = np.where(real, d.pin_offset_x[fnp][ls], 0).astype(np.float32)
    ln_offy = np.where(real, d.pin_offset_y[fnp][ls], 0).astype(np.float32)
    ln_csr = np.where(real, csr_pos[ls], 0).astype(np.int32)
    plan = (dev(g_deg.numpy()), dev(g_base.numpy()), dev(g_net.numpy()), dev(ln_node), dev(ln_offx), dev(ln_offy))
    return plan, dev(ln_csr), csr_pos, slot_of_pin, g_deg.numpy()


@pytest.mark.parametrize("weighted", [False, True])
def test_wa_lanes_against_reference(C, golden, weighted):
    """Lane-per-net WA (nets of degree <= 8 one per lane, larger nets one per
    warp): value and per-pin gradient against the reference's merged op
    (golden) or the oracle with random net weights; the HPWL of the same plan
    against the reference's HPWL."""
    g = golden("design_small.npz")
    d = small_design()
    n, P = d.num_nodes, d.num_pins
    plan, ln_csr, csr_pos, slot_of_pin, deg = lane_inputs(C, d)
    assert deg.max() > 8 and deg.min() <= 2  # both the lane and the warp paths run
    pos = g["pos"].astype(np.float32)
    xy = pack_xy(pos, n)
    mask = dev(g["net_mask"])
    weights = (np.random.RandomState(6).uniform(0.5, 2.0, d.num_nets).astype(np.float32) if weighted
               else d.net_weights.astype(np.float32))
    inv_gamma = torch.tensor([float(g["inv_gamma"])], device="cuda")
    wl = torch.zeros(1280, dtype=torch.float64, device="cuda")
    hp = torch.zeros(1280, dtype=torch.float64, device="cuda")
    gnode = torch.empty(2 * P, device="cuda")
    C.wa_lanes_forward(xy, *plan[:3], *plan[3:], ln_csr, dev(weights), mask, inv_gamma, wl, gnode, mask, hp)
    got = gnode.cpu().numpy().reshape(-1, 2)[csr_pos[slot_of_pin]]  # per pin id
    if weighted:
        ref_wl, _, ref_grad = oracle.wa_merged(g["pin_pos"], d.flat_net2pin_map, d.flat_net2pin_start_map,
                                               g["net_mask"], weights, float(g["inv_gamma"]))
        w_pin = weights[d.pin2net_map]
        exp = np.stack([ref_grad[:P] * w_pin, ref_grad[P:] * w_pin], axis=1)
    else:
        ref_wl = float(g["wa_wl"])
        exp = np.stack([g["wa_grad_intermediate"][:P], g["wa_grad_intermediate"][P:]], axis=1)
    assert math.isclose(float(wl[0].item()), ref_wl, rel_tol=1e-5)
    # the gradient bar of the merged op, scaled by the largest net weight
    np.testing.assert_allclose(got, exp, rtol=1e-5, atol=1e-6 * float(weights.max()))
    ref_hpwl = oracle.hpwl(g["pin_pos"], d.flat_net2pin_map, d.flat_net2pin_start_map, g["net_mask"], weights)
    assert math.isclose(float(hp[0].item()), ref_hpwl, rel_tol=1e-6)
    if not weighted:
        assert math.isclose(float(hp[0].item()), float(g["hpwl"]), rel_tol=1e-6)
    alone = torch.zeros(1280, dtype=torch.float64, device="cuda")
    C.hpwl_lanes(xy, *plan, dev(weights), mask, alone)
    assert alone[0].item() == hp[0].item()  # same plan, same summation order


def test_wa_lanes_net_order_invariant(C, golden):
    """The planner's net order only moves nets in memory: every pin gradient
    is bit-identical under a shuffled order (each net's loops run the same),
    the fp64 totals agree to rounding."""
    g = golden("design_small.npz")
    d = small_design()
    n, P = d.num_nodes, d.num_pins
    xy = pack_xy(g["pos"].astype(np.float32), n)
    mask = dev(g["net_mask"])
    inv_gamma = torch.tensor([float(g["inv_gamma"])], device="cuda")
    out = []
    for order in (None, np.random.RandomState(3).permutation(d.num_nets)):
        plan, ln_csr, csr_pos, slot_of_pin, _ = lane_inputs(C, d, order)
        wl = torch.zeros(1280, dtype=torch.float64, device="cuda")
        hp = torch.zeros(1280, dtype=torch.float64, device="cuda")
        gnode = torch.empty(2 * P, device="cuda")
        C.wa_lanes_forward(xy, *plan[:3], *plan[3:], ln_csr, None, mask, inv_gamma, wl, gnode, mask, hp)
        out.append((gnode.cpu().numpy().reshape(-1, 2)[csr_pos[slot_of_pin]], wl[0].item(), hp[0].item()))
    (g0, w0, h0), (g1, w1, h1) = out
    assert np.array_equal(g0, g1)
    assert math.isclose(w0, w1, rel_tol=1e-12) and math.isclose(h0, h1, rel_tol=1e-12)


def test_reference_ep_unit_case(C, golden):
    """The reference's own electric-potential unit-test case (one movable cell,
    83 fixed cells of which one spans the die width, die from y = 6, bins of
    16.34 x 11.16): fixed and density maps and the force bit-exact against the
    reference CPU op; the Poisson solve with non-square bins against the fp64
    oracle; the ElectricPotential module against the reference's energy and
    gradient.  The gradient bar follows from the field bar: the cell's force
    sums the field over its area, so |dF| <= 2 * tol * max|E| * area."""
    from dreamplace_b200.electric_potential import ElectricPotential, poisson_solve
    g = golden("ep_unit.npz")
    d = ep_unit_case(g)
    M, N, nm, nt = d.num_bins_x, d.num_bins_y, d.num_movable_nodes, d.num_terminals
    geo = (d.xl, d.yl, d.xh, d.yh, d.bin_size_x, d.bin_size_y)
    pos = dev(g["pos"])
    sx, sy, sxc, syc, ox, oy, ratio = stretched_t(d)
    bcx, bcy = dev(d.bcx), dev(d.bcy)
    snm = dev(np.arange(nm, dtype=np.int32))
    for det in (0, 1):
        fixed = C.fixed_density_map(pos, sx, sy, bcx, bcy, *geo, nm, nt, M, N, 0, 0, det)
        init = fixed.mul(d.target_density).view(-1)
        dm = C.density_map(pos, sxc, syc, ox, oy, ratio, init, init, init, d.target_density, *geo, nm, 0, 0, M, N,
                           0, 0, 0, 0, det, snm)
        ref_fixed, ref_dm = (g["%s_det%d" % (k, det)].reshape(-1) for k in ("fixed_map", "density_map"))
        if det:
            assert np.array_equal(fixed.cpu().numpy().reshape(-1), ref_fixed)
            assert np.array_equal(dm.cpu().numpy().reshape(-1), ref_dm)
        else:
            np.testing.assert_allclose(fixed.cpu().numpy().reshape(-1), ref_fixed, rtol=1e-5, atol=1e-3)
            np.testing.assert_allclose(dm.cpu().numpy().reshape(-1), ref_dm, rtol=1e-5, atol=1e-3)
    ex = dev(window_to_map(g, "field_x_window", M, N)).view(-1)
    ey = dev(window_to_map(g, "field_y_window", M, N)).view(-1)
    force = C.electric_force(torch.ones(1, device="cuda"), M, N, 0, 0, 0, 0, ex, ey, pos, sxc, syc, ox, oy, ratio,
                             pos, pos, *geo, nm, 0, 1, snm, -1.0)
    assert np.array_equal(force.cpu().numpy(), g["force"])
    dmap = g["density_map_det1"].reshape(M, N)
    rex, rey, renergy = oracle.poisson(dmap, d.bin_size_x, d.bin_size_y)
    emax = max(np.max(np.abs(rex)), np.max(np.abs(rey)))
    area = float(d.node_size_x[0] * d.node_size_y[0])
    for precision in ("fp32", "split_bf16"):
        tol = FIELD_TOL[precision]
        rho = dev(dmap).mul_(1.0 / (d.bin_size_x * d.bin_size_y))
        fx, fy, energy = poisson_solve(rho, d.bin_size_x, d.bin_size_y, precision)
        for got, ref in ((fx, rex), (fy, rey)):
            assert np.max(np.abs(got.cpu().numpy() - ref)) <= tol * np.max(np.abs(ref)), precision
        assert abs(float(energy.item()) - renergy) <= 10 * tol * abs(renergy)
        p = dev(g["pos"]).requires_grad_(True)
        op = ElectricPotential(sx, sy, bcx, bcy, d.target_density, d.xl, d.yl, d.xh, d.yh, d.bin_size_x,
                               d.bin_size_y, nm, nt, 0, 0, True, snm, precision=precision)
        e = op(p)
        assert math.isclose(float(e.item()), float(g["energy"]), rel_tol=10 * tol), precision
        e.backward()
        err = np.max(np.abs(p.grad.cpu().numpy() - g["force"]))
        assert err <= 2 * tol * emax * area, (precision, err)
        assert np.count_nonzero(p.grad.cpu().numpy()) == 2 * nm
    assert C.tc_status() == 0


@pytest.mark.parametrize("precision", ["fp32", "tf32"])
def test_transforms_reference_unit_inputs(C, golden, precision):
    """The 4 x 8 inputs of the reference's transform unit tests against the
    reference's dct2_fft2 op (bf16 operands need rows of 16 bytes, i.e. map
    sides that are multiples of 8)."""
    from dreamplace_b200 import dct2_fft2 as dct
    g = golden("dct_unit.npz")
    for cls, name, key in ((dct.DCT2, "dct2_fft2", "x"), (dct.IDCT2, "idct2_fft2", "x_int"),
                           (dct.IDCT_IDXST, "idct_idxst", "x_int"), (dct.IDXST_IDCT, "idxst_idct", "x_int")):
        got = cls(precision=precision)(dev(g[key])).cpu().numpy()
        ref = g[name]
        assert np.max(np.abs(got - ref)) <= FIELD_TOL[precision] * np.max(np.abs(ref)), (name, precision)
    assert C.tc_status() == 0


def test_wa_edge_nets(C, golden):
    """Edge-case nets against the reference's merged WA and HPWL ops: degree-1
    nets (kept by the mask, zero wirelength and gradient), partial lane groups
    of every degree 2..8, warp nets of degree 9..300, coincident pins, a net
    spread far beyond gamma (exp underflow), masked and weighted nets; through
    the drop-in op and through the engine's lane kernel.  With pins hundreds of
    gamma apart the gradient is a small difference of large terms, so the bar
    on each pin is relative to those terms (wa_cancellation_scale): CUDA's and
    glibc's expf differ by an ulp here and there, which moves such a gradient
    by ~2e-7 of the scale (measured on the CPU with a one-ulp perturbation)."""
    g = golden("wa_edge.npz")
    d = wa_edge_netlist(g)
    P, n = d.num_pins, d.num_nodes
    pin = dev(g["pin_pos"])
    flat, start, p2n = dev(g["flat_netpin"]), dev(g["netpin_start"]), dev(g["pin2net"])
    w, mask = dev(g["net_weights"]), dev(g["net_mask"])
    ig = float(np.float32(1.0) / g["gamma"])
    inv_gamma = torch.tensor([ig], device="cuda")
    assert np.array_equal(C.pin_pos_forward(dev(g["pos"]), dev(g["pin_offset_x"]), dev(g["pin_offset_y"]),
                                            dev(g["pin2node"])).cpu().numpy(), g["pin_pos"])
    scale = wa_cancellation_scale(g["pin_pos"], g["flat_netpin"], g["netpin_start"], g["net_mask"], ig)
    w_pin2 = np.tile(g["net_weights"][g["pin2net"]], 2)

    def check(got, ref, weight=1.0):
        bar = 1e-6 + 1e-5 * np.abs(ref) + 4e-6 * scale * weight
        assert np.all(np.abs(got - ref) <= bar), float(np.max(np.abs(got - ref) - bar))

    wl, gi = C.wa_merged_forward(pin, flat, start, p2n, w, mask, inv_gamma)
    assert math.isclose(float(wl.item()), float(g["wl"]), rel_tol=1e-5)
    check(gi.cpu().numpy(), g["grad_intermediate"])
    out = C.wa_merged_backward(torch.ones(1, device="cuda"), pin, gi.clone(), flat, start, p2n, w, mask, inv_gamma,
                               None)
    check(out.cpu().numpy(), g["grad"], w_pin2)
    deg = np.diff(g["netpin_start"])
    one = g["flat_netpin"][g["netpin_start"][:-1][deg == 1]]
    assert not np.any(gi.cpu().numpy()[np.r_[one, P + one]])  # degree-1 nets: zero gradient
    h = C.hpwl_forward(pin, flat, start, w, dev(g["hpwl_mask"]))
    assert math.isclose(float(h.item()), float(g["hpwl"]), rel_tol=1e-6)
    # the engine's lane kernel (node positions + pin offsets, lane groups by degree)
    plan, ln_csr, csr_pos, slot_of_pin, g_deg = lane_inputs(C, d)
    assert set(range(1, 9)) <= set(g_deg.tolist()) and g_deg.max() == 300
    xy = pack_xy(g["pos"], n)
    wl2 = torch.zeros(1280, dtype=torch.float64, device="cuda")
    hp = torch.zeros(1280, dtype=torch.float64, device="cuda")
    gnode = torch.empty(2 * P, device="cuda")
    C.wa_lanes_forward(xy, *plan, ln_csr, w, mask, inv_gamma, wl2, gnode, dev(g["hpwl_mask"]), hp)
    got = gnode.cpu().numpy().reshape(-1, 2)[csr_pos[slot_of_pin]]
    check(np.concatenate([got[:, 0], got[:, 1]]), g["grad_intermediate"] * w_pin2, w_pin2)
    assert math.isclose(float(wl2[0].item()), float(g["wl"]), rel_tol=1e-5)
    assert math.isclose(float(hp[0].item()), float(g["hpwl"]), rel_tol=1e-6)


def test_boundary_and_wide_cells(C):
    """Cells on, across and beyond every die edge and corner, movable cells 5
    and 9 bins wide and 6 bins tall (the per-bin paths of the window scatter
    and of the field gather), fillers across the edge, a filler-only pass and
    an empty pass: the order-driven scatter's integer map and the field
    gather's force bit-exact with the oracle (which clamps bin ranges as the
    reference CPU op does)."""
    d = synthetic.scaled(3000, num_bins=64, seed=7, name="edge_cells")
    n, m, nf = d.num_nodes, d.num_movable_nodes, d.num_filler_nodes
    bsx, bsy = d.bin_size_x, d.bin_size_y
    sx, sy = d.node_size_x.copy(), d.node_size_y.copy()
    sx[:50] = 5 * bsx
    sx[50:100] = 9 * bsx
    sy[100:150] = 6 * bsy
    d.node_size_x, d.node_size_y = sx.astype(np.float32), sy.astype(np.float32)
    rng = np.random.RandomState(4)
    pos = d.initial_positions().astype(np.float64)
    pos[:m] = rng.uniform(d.xl, d.xh, m)
    pos[n:n + m] = rng.uniform(d.yl, d.yh, m)
    X, Y = pos[:n], pos[n:]
    X[150:200] = d.xl
    Y[200:250] = d.yl
    X[250:300] = d.xh - sx[250:300]
    Y[300:350] = d.yh - sy[300:350]
    X[350:400] = d.xl - 0.5 * sx[350:400]
    X[400:450] = d.xh - 0.3 * sx[400:450]
    Y[450:500] = d.yl - 0.7 * sy[450:500]
    Y[500:550] = d.yh - 0.2 * sy[500:550]
    X[550:600] = d.xl - 10 * bsx
    X[600:650] = d.xh + 3 * bsx
    X[650:700], Y[650:700] = d.xl - 0.5 * sx[650:700], d.yh - 0.5 * sy[650:700]
    X[700:750], Y[700:750] = d.xh - 0.5 * sx[700:750], d.yl - 0.5 * sy[700:750]
    X[0:20] = d.xh - 2 * bsx  # wide cells across the right edge
    Y[100:120] = d.yl - 2 * bsy  # tall cells across the bottom edge
    f0 = n - nf
    X[f0:f0 + 50] = d.xh - 0.5 * sx[f0:f0 + 50]
    Y[f0 + 50:f0 + 100] = d.yh - 0.5 * sy[f0 + 50:f0 + 100]
    pos = pos.astype(np.float32)
    s = oracle.stretched(d.node_size_x, d.node_size_y, bsx, bsy)
    geo = (d.xl, d.yl, d.xh, d.yh, bsx, bsy, d.num_bins_x, d.num_bins_y)
    nb = d.num_bins_x * d.num_bins_y
    xy = pack_xy(pos, n)
    idx = np.r_[0:m, f0:n].astype(np.int32)
    fx = dev(np.random.RandomState(5).standard_normal(nb).astype(np.float32))
    fy = dev(np.random.RandomState(6).standard_normal(nb).astype(np.float32))
    ref_force = oracle.electric_force(fx.cpu().numpy(), fy.cpu().numpy(), pos, *s, n, m, nf, d.num_bins_x,
                                      d.num_bins_y, d.xl, d.yl, bsx, bsy)
    cases = (("all", idx, m), ("fillers", idx[m:], 0), ("empty", idx, 0))
    for name, order, num_mov in cases:
        if name == "all":
            order = np.r_[spatial_order(d, pos, idx[:m]), spatial_order(d, pos, idx[m:])].astype(np.int32)
        count = 0 if name == "empty" else len(order)
        ref_map, ref_fx = oracle.triangle_density_map(pos, *s, n, num_mov, nf if count else 0, d.num_bins_x,
                                                      d.num_bins_y, d.xl, d.yl, d.xh, d.yh, bsx, bsy,
                                                      deterministic=True)
        rec4, ratio_o, _ = records(C, d, order)
        out = torch.empty(nb, device="cuda")
        scratch = torch.empty(nb, dtype=torch.int64, device="cuda")
        C.density_map_ordered_into(order_xy(C, xy, order), rec4, ratio_o, count, None, *geo, 1, scratch, out)
        assert np.array_equal(scratch.cpu().numpy(), ref_fx), name
        assert np.array_equal(out.cpu().numpy(), ref_map), name
        if count:
            force_o = torch.empty(2 * len(order), device="cuda")
            C.electric_force_ordered(torch.ones(1, device="cuda"), fx, fy, order_xy(C, xy, order), rec4, ratio_o,
                                     count, d.xl, d.yl, bsx, bsy, d.num_bins_x, d.num_bins_y, -1.0, force_o)
            fo = force_o.cpu().numpy().reshape(-1, 2)
            assert np.array_equal(fo[:, 0], ref_force[order]), name
            assert np.array_equal(fo[:, 1], ref_force[n + order]), name
    # the drop-in ops (node order, thread per cell) on the same cells
    _, _, sxc, syc, ox, oy, ratio = stretched_t(d)
    tpos = dev(pos)
    ref_map, ref_fx = oracle.triangle_density_map(pos, *s, n, m, nf, d.num_bins_x, d.num_bins_y, d.xl, d.yl, d.xh,
                                                  d.yh, bsx, bsy, deterministic=True)
    fxm = C.density_map_fixed_point(tpos, sxc, syc, ox, oy, ratio, d.xl, d.yl, d.xh, d.yh, bsx, bsy, m, nf,
                                    d.num_bins_x, d.num_bins_y, sorted_map(d))
    assert np.array_equal(fxm.cpu().numpy(), ref_fx)
    force = C.electric_force(torch.ones(1, device="cuda"), d.num_bins_x, d.num_bins_y, 0, 0, 0, 0, fx, fy, tpos, sxc,
                             syc, ox, oy, ratio, tpos, tpos, d.xl, d.yl, d.xh, d.yh, bsx, bsy, m, nf, 1,
                             sorted_map(d), -1.0)
    assert np.array_equal(force.cpu().numpy(), ref_force)
    # the cells entirely outside the die contribute nothing and feel no force
    assert not np.any(ref_force[np.r_[550:650]])


def test_electric_potential_options(C, golden):
    """The reference module's options against the reference ops composed as
    its module does (ep_options.npz): movable-macro ratios at target density
    0.8 and padding 2 give the same density map bit for bit (deterministic),
    the energy and gradient of the fp32 solve; fast_mode returns zero energy
    and the same gradient bit for bit; overflow mode and the ElectricOverflow
    module (movable cells only) give the reference's overflow and max density."""
    from dreamplace_b200.electric_potential import ElectricOverflow, ElectricPotential
    g = golden("ep_options.npz")
    d = small_design()
    pos_np = golden("design_small.npz")["pos"]
    target, padding = float(g["target_density"]), int(g["padding"])
    mask = dev(g["macro_mask"]).bool()
    bcx, bcy = dev(d.bin_centers(d.xl, d.xh, d.bin_size_x)), dev(d.bin_centers(d.yl, d.yh, d.bin_size_y))
    args = (dev(d.node_size_x), dev(d.node_size_y), bcx, bcy, target, d.xl, d.yl, d.xh, d.yh, d.bin_size_x,
            d.bin_size_y, d.num_movable_nodes, d.num_terminals)
    grads = []
    for fast in (False, True):
        op = ElectricPotential(*args, d.num_filler_nodes, padding, True, sorted_map(d), movable_macro_mask=mask,
                               fast_mode=fast, precision="fp32")
        p = dev(pos_np).requires_grad_(True)
        e = op(p)
        if fast:
            assert float(e.item()) == 0.0
        else:
            assert math.isclose(float(e.item()), float(g["energy"]), rel_tol=1e-4)
            dm = op._density_map(p.detach(), d.num_filler_nodes)
            assert np.array_equal(dm.cpu().numpy(), g["density_map"])
        e.backward()
        grads.append(p.grad.clone())
        ovf, mx = op(p.detach(), mode="overflow")
        assert math.isclose(float(ovf), float(g["overflow"]), rel_tol=1e-5)
        assert math.isclose(float(mx), float(g["max_density"]), rel_tol=1e-6)
    ref = g["force"]
    assert np.max(np.abs(grads[0].cpu().numpy() - ref)) <= 1e-4 * np.max(np.abs(ref))
    assert torch.equal(grads[0], grads[1])
    ov = ElectricOverflow(*args, 0, padding, True, sorted_map(d), movable_macro_mask=mask)
    ovf, mx = ov(dev(pos_np))
    assert math.isclose(float(ovf.item()), float(g["overflow"]), rel_tol=1e-5)
    assert math.isclose(float(mx.item()), float(g["max_density"]), rel_tol=1e-6)
