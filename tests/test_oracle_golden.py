"""The CPU oracle against the reference CPU ops' outputs (tests/golden)."""
import math

import numpy as np

import oracle
from dreamplace_b200 import synthetic


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
