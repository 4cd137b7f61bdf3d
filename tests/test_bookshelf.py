"""Bookshelf round trip of a synthetic design: the netlist, geometry, and the
derived fillers / target density survive write + read."""
import numpy as np

from dreamplace_b200 import bookshelf, synthetic


def test_round_trip(tmp_path):
    d = synthetic.cells_10k()
    aux = bookshelf.write_bookshelf(d, str(tmp_path))
    r = bookshelf.read_bookshelf(aux, num_bins=d.num_bins_x)
    assert (r.num_movable_nodes, r.num_terminals, r.num_nets, r.num_pins) == \
        (d.num_movable_nodes, d.num_terminals, d.num_nets, d.num_pins)
    assert (r.xl, r.yl, r.xh, r.yh) == (d.xl, d.yl, d.xh, d.yh)
    np.testing.assert_array_equal(r.node_size_x[:d.num_physical_nodes], d.node_size_x[:d.num_physical_nodes])
    np.testing.assert_array_equal(r.pin2node_map, d.pin2node_map)
    np.testing.assert_array_equal(r.flat_net2pin_start_map, d.flat_net2pin_start_map)
    np.testing.assert_allclose(r.pin_offset_x, d.pin_offset_x, atol=1e-5)
    np.testing.assert_allclose(r.pin_offset_y, d.pin_offset_y, atol=1e-5)
    np.testing.assert_allclose(r.node_x[d.num_movable_nodes:], d.node_x[d.num_movable_nodes:])
    assert r.num_filler_nodes == d.num_filler_nodes and r.target_density == d.target_density
