"""Synthetic design generator: sizes, degree law and the reference's filler rule."""
import numpy as np

from dreamplace_b200 import synthetic


def test_10k_design_shapes():
    d = synthetic.cells_10k()
    assert d.num_movable_nodes == 10000 and d.num_terminals == 50
    assert d.num_nets == 10200 and d.num_bins_x == 128
    deg = np.diff(d.flat_net2pin_start_map)
    assert deg.min() >= 2 and deg.max() <= 50
    assert abs(deg.mean() - 3.22) < 0.1
    assert d.flat_net2pin_start_map[-1] == d.num_pins
    assert np.all(d.node_size_x[:10000] >= 2) and np.all(d.node_size_x[:10000] <= 32)
    # fillers: round(max(space*t - movable, 0) / (w*h))
    fw, fh = d.extra["filler_size"]
    exp = int(round(max(d.total_space_area * d.target_density - d.total_movable_node_area, 0) / (fw * fh)))
    assert d.num_filler_nodes == exp
    # macros inside the die, no overlap
    m = d.num_movable_nodes
    x, y = d.node_x[m:], d.node_y[m:]
    w, h = d.node_size_x[m:m + 50], d.node_size_y[m:m + 50]
    assert np.all(x >= 0) and np.all(x + w <= 3000) and np.all(y + h <= 3000)
    for i in range(50):
        ov = (x[i] < x + w) & (x < x[i] + w[i]) & (y[i] < y + h) & (y < y[i] + h[i])
        assert ov.sum() == 1


def test_csr_consistency():
    d = synthetic.scaled(5000, seed=3)
    p = np.arange(d.num_pins)
    assert np.array_equal(np.sort(d.flat_node2pin_map), p)
    nodes = np.repeat(np.arange(d.num_physical_nodes), np.diff(d.flat_node2pin_start_map))
    assert np.array_equal(d.pin2node_map[d.flat_node2pin_map], nodes)
    nets = np.repeat(np.arange(d.num_nets), np.diff(d.flat_net2pin_start_map))
    assert np.array_equal(d.pin2net_map[d.flat_net2pin_map], nets)


def test_initial_positions_reference_rule():
    d = synthetic.cells_10k()
    pos = d.initial_positions()
    n, m = d.num_nodes, d.num_movable_nodes
    assert abs(pos[:m].mean() - 1500) < 1 and pos[:m].std() < 5
    assert np.all(pos[d.num_physical_nodes:n] <= d.xh - d.node_size_x[-1])
    assert np.array_equal(pos[m:d.num_physical_nodes], d.node_x[m:])


def test_batch_partition_and_bins():
    """Batched placement: every design lands on exactly one rank; bins follow
    the nearest power of two of sqrt(cells), clamped to 64..512."""
    from dreamplace_b200 import batch
    for world in (1, 2, 3, 8):
        seen = sorted(i for r in range(world) for i in batch.assign(64, r, world))
        assert seen == list(range(64))
    assert batch.bins_for(5000) == 64 and batch.bins_for(20000) == 128 and batch.bins_for(200000) == 512
    ds = batch.batch_set(3, seed=2, lo=5000, hi=8000)
    assert [d.name for d in ds] == ["batch0", "batch1", "batch2"]
    assert all(5000 <= d.num_movable_nodes <= 8000 and d.num_bins_x == 64 for d in ds)
