"""The drop-in ops have no CPU path: CPU tensors raise RuntimeError (the
reference ops' device checks raise the same way) instead of falling back to
another implementation.  Runs without a GPU."""
import numpy as np
import pytest
import torch

from dreamplace_b200 import synthetic


def small():
    return synthetic.scaled(3000, num_bins=64, seed=7, name="golden_small")


def test_transforms_reject_cpu_maps():
    from dreamplace_b200.dct2_fft2 import DCT2, IDCT2, IDCT_IDXST, IDXST_IDCT
    for cls in (DCT2, IDCT2, IDCT_IDXST, IDXST_IDCT):
        with pytest.raises(RuntimeError, match="CUDA only"):
            cls()(torch.zeros(8, 8))


def test_electric_potential_rejects_cpu_positions():
    from dreamplace_b200.electric_potential import ElectricPotential
    d = small()
    t = torch.from_numpy
    op = ElectricPotential(t(d.node_size_x), t(d.node_size_y), t(d.bin_centers(d.xl, d.xh, d.bin_size_x)),
                           t(d.bin_centers(d.yl, d.yh, d.bin_size_y)), d.target_density, d.xl, d.yl, d.xh, d.yh,
                           d.bin_size_x, d.bin_size_y, d.num_movable_nodes, d.num_terminals, d.num_filler_nodes, 0,
                           False, None)
    op.initial_density_map = torch.zeros(d.num_bins_x, d.num_bins_y)  # skip the fixed-map set-up
    with pytest.raises(RuntimeError, match="CUDA only"):
        op(t(d.initial_positions()), mode="overflow")


def test_wirelength_and_pins_reject_cpu_positions():
    from dreamplace_b200.placement_ops import PinPos
    from dreamplace_b200.weighted_average_wirelength import WeightedAverageWirelength
    d = small()
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a))  # noqa: E731
    deg = np.diff(d.flat_net2pin_start_map)
    wa = WeightedAverageWirelength(t(d.flat_net2pin_map), t(d.flat_net2pin_start_map), t(d.pin2net_map),
                                   t(d.net_weights), t((deg >= 2).astype(np.uint8)),
                                   torch.zeros(d.num_pins, dtype=torch.bool), torch.tensor([10.0]))
    with pytest.raises(RuntimeError, match="CUDA only"):
        wa(torch.zeros(2 * d.num_pins))
    pp = PinPos(t(d.pin_offset_x), t(d.pin_offset_y), t(d.pin2node_map), t(d.flat_node2pin_map),
                t(d.flat_node2pin_start_map), d.num_physical_nodes)
    with pytest.raises(RuntimeError, match="CUDA only"):
        pp(t(d.initial_positions()))
