"""The CPU oracle against the reference CPU ops' outputs (tests/golden)."""
import math

import numpy as np

import oracle
from dreamplace_b200 import synthetic
from golden_cases import ep_unit_case, window_to_map


def small_design():
    return synthetic.scaled(3000, num_bins=64, seed=7, name="golden_small")


def test_wa_unit_golden(golden):
    g = golden("wa_unit.npz")
    wl, partial, grad = oracle.wa_merged(g["pos"], g["flat_netpin"], g["netpin_start"], g["net_mask"],
                                         g["net_weights"], float(np.float32(1.0) / g["gamma"]))
    assert abs(wl - float(g["wl"])) <= 1e-6 * max(1.0, abs(float(g["wl"])))
    np.testing.assert_allclose(grad, g["grad_intermediate"], rtol=1e-6, atol=1e-7)


def test_dct_oracle_golden(golden):
    g = golden("dct_small.npz")
    x = g["x"]
    for name, f in (("dct2_fft2", oracle.dct2), ("idct2_fft2", oracle.idct2), ("idct_idxst", oracle.idct_idxst),
                    ("idxst_idct", oracle.idxst_idct)):
        ref = g[name].astype(np.float64)
        got = f(x)
        assert np.max(np.abs(got - ref)) <= 2e-6 * max(1.0, np.max(np.abs(ref))), name


def _stretched(d):
    return oracle.stretched(d.node_size_x, d.node_size_y, d.bin_size_x, d.bin_size_y)


def test_density_maps_bit_exact(golden):
    g = golden("design_small.npz")
    d = small_design()
    pos = g["pos"]
    bcx = d.bin_centers(d.xl, d.xh, d.bin_size_x)
    bcy = d.bin_centers(d.yl, d.yh, d.bin_size_y)
    for det in (False, True):
        fixed = oracle.fixed_density_map(pos, d.node_size_x, d.node_size_y, bcx, bcy, d.num_nodes,
                                         d.num_movable_nodes, d.num_terminals, d.num_bins_x, d.num_bins_y, d.xl,
                                         d.yl, d.xh, d.yh, d.bin_size_x, d.bin_size_y, deterministic=det)
        assert np.array_equal(fixed.reshape(-1), g["fixed_map_det%d" % int(det)].reshape(-1))
        init = (fixed * np.float32(d.target_density)).astype(np.float32)
        sxc, syc, ox, oy, ratio = _stretched(d)
        dm, fx = oracle.triangle_density_map(pos, sxc, syc, ox, oy, ratio, d.num_nodes, d.num_movable_nodes,
                                             d.num_filler_nodes, d.num_bins_x, d.num_bins_y, d.xl, d.yl, d.xh, d.yh,
                                             d.bin_size_x, d.bin_size_y, initial=init, deterministic=det)
        ref = g["density_map_det%d" % int(det)].reshape(-1)
        if det:
            assert np.array_equal(dm, ref)
        else:
            np.testing.assert_allclose(dm, ref, rtol=1e-5, atol=1e-3)


def test_force_bit_exact(golden):
    g = golden("design_small.npz")
    d = small_design()
    sxc, syc, ox, oy, ratio = _stretched(d)
    f = oracle.electric_force(g["field_x"].reshape(-1), g["field_y"].reshape(-1), g["pos"], sxc, syc, ox, oy, ratio,
                              d.num_nodes, d.num_movable_nodes, d.num_filler_nodes, d.num_bins_x, d.num_bins_y,
                              d.xl, d.yl, d.bin_size_x, d.bin_size_y)
    assert np.array_equal(f, g["force"])


def test_poisson_oracle_against_reference_fft(golden):
    g = golden("design_small.npz")
    d = small_design()
    ex, ey, energy = oracle.poisson(g["density_map_det1"].reshape(d.num_bins_x, d.num_bins_y), d.bin_size_x,
                                    d.bin_size_y)
    for got, ref in ((ex, g["field_x"]), (ey, g["field_y"])):
        assert np.max(np.abs(got - ref)) <= 1e-4 * np.max(np.abs(ref))
    assert math.isclose(energy, float(g["energy"]), rel_tol=1e-4)


def test_pins_nets(golden):
    g = golden("design_small.npz")
    d = small_design()
    pin = oracle.pin_pos(g["pos"], d.pin_offset_x, d.pin_offset_y, d.pin2node_map, d.num_nodes)
    assert np.array_equal(pin, g["pin_pos"])
    back = oracle.pin_pos_backward(g["pin_grad_in"], d.flat_node2pin_map, d.flat_node2pin_start_map,
                                   d.num_physical_nodes, d.num_nodes)
    assert np.array_equal(back, g["pin_pos_backward"])
    wl, partial, grad = oracle.wa_merged(pin, d.flat_net2pin_map, d.flat_net2pin_start_map, g["net_mask"],
                                         d.net_weights, float(g["inv_gamma"]))
    assert math.isclose(wl, float(g["wa_wl"]), rel_tol=1e-5)
    np.testing.assert_allclose(grad, g["wa_grad_intermediate"], rtol=1e-5, atol=1e-6)
    deg = np.diff(d.flat_net2pin_start_map)
    h = oracle.hpwl(pin, d.flat_net2pin_map, d.flat_net2pin_start_map, (deg >= 2).astype(np.uint8), d.net_weights)
    assert math.isclose(h, float(g["hpwl"]), rel_tol=1e-5)


def test_ep_unit_case_oracle(golden):
    """The reference's own electric-potential unit-test case (one movable cell,
    83 fixed cells of which one spans the die width, die starting at y = 6,
    non-power-of-two bin sizes): maps and force bit-exact, Poisson energy within
    the fp32 FFT's rounding."""
    g = golden("ep_unit.npz")
    d = ep_unit_case(g)
    xl, yl, xh, yh, M, N = d.xl, d.yl, d.xh, d.yh, d.num_bins_x, d.num_bins_y
    bsx, bsy, n, m, nt = d.bin_size_x, d.bin_size_y, d.num_nodes, d.num_movable_nodes, d.num_terminals
    bcx, bcy = d.bcx, d.bcy
    s = oracle.stretched(g["node_size_x"], g["node_size_y"], bsx, bsy)
    for det in (False, True):
        fixed = oracle.fixed_density_map(g["pos"], g["node_size_x"], g["node_size_y"], bcx, bcy, n, m, nt, M, N, xl,
                                         yl, xh, yh, bsx, bsy, deterministic=det)
        ref_fixed = g["fixed_map_det%d" % int(det)].reshape(-1)
        init = (fixed * np.float32(float(g["target_density"]))).astype(np.float32)
        dm, _ = oracle.triangle_density_map(g["pos"], *s, n, m, 0, M, N, xl, yl, xh, yh, bsx, bsy, initial=init,
                                            deterministic=det)
        ref_dm = g["density_map_det%d" % int(det)].reshape(-1)
        if det:
            assert np.array_equal(fixed.reshape(-1), ref_fixed) and np.array_equal(dm, ref_dm)
        else:
            np.testing.assert_allclose(fixed.reshape(-1), ref_fixed, rtol=1e-5, atol=1e-3)
            np.testing.assert_allclose(dm, ref_dm, rtol=1e-5, atol=1e-3)
    ex, ey = window_to_map(g, "field_x_window", M, N), window_to_map(g, "field_y_window", M, N)
    f = oracle.electric_force(ex.reshape(-1), ey.reshape(-1), g["pos"], *s, n, m, 0, M, N, xl, yl, bsx, bsy)
    assert np.array_equal(f, g["force"])
    assert np.count_nonzero(f) == 2 * m  # fixed cells get no force
    oex, oey, energy = oracle.poisson(g["density_map_det1"].reshape(M, N), bsx, bsy)
    k0, k1, h0, h1 = (int(v) for v in g["field_window"])
    for got, ref in ((oex[k0:k1, h0:h1], g["field_x_window"]), (oey[k0:k1, h0:h1], g["field_y_window"])):
        assert np.max(np.abs(got - ref)) <= 1e-4 * np.max(np.abs(ref))
    assert math.isclose(energy, float(g["energy"]), rel_tol=1e-4)


def test_dct_unit_oracle(golden):
    """The 4 x 8 inputs of the reference's transform unit tests."""
    g = golden("dct_unit.npz")
    for name, f, x in (("dct2_fft2", oracle.dct2, g["x"]), ("idct2_fft2", oracle.idct2, g["x_int"]),
                       ("idct_idxst", oracle.idct_idxst, g["x_int"]), ("idxst_idct", oracle.idxst_idct, g["x_int"])):
        ref = g[name].astype(np.float64)
        assert np.max(np.abs(f(x) - ref)) <= 2e-6 * max(1.0, np.max(np.abs(ref))), name


def test_wa_edge_nets_oracle(golden):
    """Degree-1 nets, partial lane groups, degrees up to 300, coincident pins,
    exp underflow, masked and weighted nets: the C restatement against the
    reference's pin_pos, merged WA and HPWL ops."""
    g = golden("wa_edge.npz")
    n = len(g["pos"]) // 2
    pin = oracle.pin_pos(g["pos"], g["pin_offset_x"], g["pin_offset_y"], g["pin2node"], n)
    assert np.array_equal(pin, g["pin_pos"])
    wl, partial, grad = oracle.wa_merged(pin, g["flat_netpin"], g["netpin_start"], g["net_mask"], g["net_weights"],
                                         float(np.float32(1.0) / g["gamma"]))
    assert math.isclose(wl, float(g["wl"]), rel_tol=1e-6)
    np.testing.assert_allclose(grad, g["grad_intermediate"], rtol=1e-6, atol=1e-6)
    deg = np.diff(g["netpin_start"])
    assert deg.min() == 1 and deg.max() == 300 and np.all(partial[(deg == 1)] == 0)
    h = oracle.hpwl(pin, g["flat_netpin"], g["netpin_start"], g["hpwl_mask"], g["net_weights"])
    assert math.isclose(h, float(g["hpwl"]), rel_tol=1e-6)


def test_ep_options_oracle(golden):
    """The reference module's options on the 3,000-cell design (movable-macro
    ratio at target density 0.8, padding 2): density map and force bit-exact
    with the oracle, overflow and max density as the reference computes them."""
    g = golden("ep_options.npz")
    d = small_design()
    pos = golden("design_small.npz")["pos"]
    n, m, nf, M, N = d.num_nodes, d.num_movable_nodes, d.num_filler_nodes, d.num_bins_x, d.num_bins_y
    target, padding = float(g["target_density"]), int(g["padding"])
    sxc, syc, ox, oy, ratio = _stretched(d)
    ratio = ratio.copy()
    ratio[:m][g["macro_mask"].astype(bool)] = np.float32(target)
    bcx = d.bin_centers(d.xl, d.xh, d.bin_size_x)
    bcy = d.bin_centers(d.yl, d.yh, d.bin_size_y)
    fixed = oracle.fixed_density_map(pos, d.node_size_x, d.node_size_y, bcx, bcy, n, m, d.num_terminals, M, N, d.xl,
                                     d.yl, d.xh, d.yh, d.bin_size_x, d.bin_size_y, deterministic=True)
    init = (fixed * np.float32(target)).astype(np.float32)
    pad = np.ones((M, N), bool)
    pad[padding:M - padding, padding:N - padding] = False
    fill = np.float32(target * d.bin_size_x * d.bin_size_y)
    for key, num_filler in (("density_map", nf), ("overflow_map", 0)):
        dm, _ = oracle.triangle_density_map(pos, sxc, syc, ox, oy, ratio, n, m, num_filler, M, N, d.xl, d.yl, d.xh,
                                            d.yh, d.bin_size_x, d.bin_size_y, initial=init, deterministic=True)
        dm = dm.reshape(M, N)
        dm[pad] = fill
        assert np.array_equal(dm, g[key]), key
    f = oracle.electric_force(g["field_x"].reshape(-1), g["field_y"].reshape(-1), pos, sxc, syc, ox, oy, ratio, n, m,
                              nf, M, N, d.xl, d.yl, d.bin_size_x, d.bin_size_y)
    assert np.array_equal(f, g["force"])
    om = g["overflow_map"].astype(np.float64)
    ba = d.bin_size_x * d.bin_size_y
    assert math.isclose(np.clip(om - target * ba, 0, None).sum(), float(g["overflow"]), rel_tol=1e-5)
    assert math.isclose(om.max() / ba, float(g["max_density"]), rel_tol=1e-6)


def test_ops_unit_golden(golden):
    """The reference's own unit-test cases of hpwl, pin_pos and move_boundary
    (unittest/ops/{hpwl,pin_pos,move_boundary}_unittest.py) as its CPU ops
    computed them: the oracle agrees bit for bit (HPWL: to the float32 the
    reference returns)."""
    g = golden("ops_unit.npz")
    h = oracle.hpwl(g["hpwl_pin_pos"], g["hpwl_flat_netpin"], g["hpwl_netpin_start"], g["hpwl_net_mask"],
                    g["hpwl_net_weights"])
    # the reference returns its total as float32; the oracle sums in fp64
    assert math.isclose(h, float(g["hpwl"]), rel_tol=1e-6)
    n = len(g["pp_pos"]) // 2
    pin = oracle.pin_pos(g["pp_pos"], g["pp_offset_x"], g["pp_offset_y"], g["pp_pin2node"], n)
    assert np.array_equal(pin, g["pin_pos"])
    back = oracle.pin_pos_backward(np.ones(2 * len(g["pp_pin2node"]), np.float32), g["pp_flat_node2pin"],
                                   g["pp_node_start"], int(g["pp_num_physical"]), n)
    assert np.array_equal(back, g["pin_pos_backward"])
    moved = oracle.move_boundary(g["mb_pos"], g["mb_node_size_x"], g["mb_node_size_y"], *g["mb_box"],
                                 int(g["mb_num_movable"]), int(g["mb_num_filler"]))
    assert np.array_equal(moved, g["move_boundary"])
