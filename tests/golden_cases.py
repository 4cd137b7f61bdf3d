"""Shared readers of the reference unit-test fixtures (tests/golden/*.npz)."""
from types import SimpleNamespace

import numpy as np


def bin_centers(lo, hi, size, n):
    """Bin centres as dreamplace/PlaceDB.py:331-345 computes them (float32)."""
    c = np.zeros(n, np.float32)
    for i in range(n):
        bl = lo + i * size
        c[i] = (bl + min(bl + size, hi)) / 2
    return c


def ep_unit_case(g):
    """The reference's electric-potential unit-test case (ep_unit.npz) as a
    design-like namespace: geometry, node counts, sizes and bin centres."""
    xl, yl, xh, yh = (float(v) for v in g["geometry"])
    M, N = (int(v) for v in g["bins"])
    bsx, bsy = (xh - xl) / M, (yh - yl) / N
    n = len(g["node_size_x"])
    return SimpleNamespace(xl=xl, yl=yl, xh=xh, yh=yh, num_bins_x=M, num_bins_y=N, bin_size_x=bsx, bin_size_y=bsy,
                           num_nodes=n, num_movable_nodes=int(g["num_movable"]),
                           num_terminals=int(g["num_terminals"]), num_filler_nodes=0,
                           node_size_x=g["node_size_x"], node_size_y=g["node_size_y"],
                           target_density=float(g["target_density"]), bcx=bin_centers(xl, xh, bsx, M),
                           bcy=bin_centers(yl, yh, bsy, N))


def window_to_map(g, key, M, N):
    """A field map that holds the fixture's window around the movable cell and
    zeros elsewhere (the force reads only bins inside the window)."""
    k0, k1, h0, h1 = (int(v) for v in g["field_window"])
    out = np.zeros((M, N), np.float32)
    out[k0:k1, h0:h1] = g[key]
    return out


def wa_edge_netlist(g):
    """The edge-case netlist (wa_edge.npz) with the attribute names of a
    synthetic design's pin/net arrays."""
    P = len(g["flat_netpin"])
    return SimpleNamespace(num_pins=P, num_nodes=len(g["pos"]) // 2, num_nets=len(g["netpin_start"]) - 1,
                           flat_net2pin_map=g["flat_netpin"], flat_net2pin_start_map=g["netpin_start"],
                           flat_node2pin_map=g["flat_node2pin"], flat_node2pin_start_map=g["node_start"],
                           pin2node_map=g["pin2node"], pin2net_map=g["pin2net"], pin_offset_x=g["pin_offset_x"],
                           pin_offset_y=g["pin_offset_y"])


def wa_cancellation_scale(pin_pos, flat_netpin, netpin_start, net_mask, inv_gamma):
    """Per pin (x then y), the size of the two terms whose difference is the
    WA gradient: (|a+| + |b+ x|) e+ + (|a-| + |b- x|) e-, with the merged
    op's a and b terms (dreamplace/ops/weighted_average_wirelength/src/
    weighted_average_wirelength_merged.cpp:89-111), in fp64.  Where x / gamma
    is large these terms are far larger than the gradient, and a one-ulp
    difference of an exponential moves the gradient by ~eps times this scale."""
    P = len(pin_pos) // 2
    T = np.zeros(2 * P)
    start = np.asarray(netpin_start, np.int64)
    deg = np.diff(start)
    live = (np.asarray(net_mask) != 0) & (deg > 0)
    if not live.any() or P == 0:
        return T
    flat = np.asarray(flat_netpin, np.int64)
    net_of_slot = np.repeat(np.arange(len(deg)), deg)
    keep = live[net_of_slot]
    idx = np.full(len(deg), -1, np.int64)
    idx[live] = np.arange(live.sum())
    k = idx[net_of_slot[keep]]
    # segments of the live nets' slots (nets stay contiguous among the kept slots)
    seg = np.r_[0, np.cumsum(deg[live])[:-1]]
    for off in (0, P):
        xs = pin_pos[off + flat[keep]].astype(np.float64)
        xmax = np.maximum.reduceat(xs, seg)
        xmin = np.minimum.reduceat(xs, seg)
        ep = np.exp((xs - xmax[k]) * inv_gamma)
        en = np.exp((xmin[k] - xs) * inv_gamma)
        s_p, s_n = np.add.reduceat(ep, seg), np.add.reduceat(en, seg)
        sx_p, sx_n = np.add.reduceat(xs * ep, seg), np.add.reduceat(xs * en, seg)
        b_p, b_n = inv_gamma / s_p, -inv_gamma / s_n
        a_p = (1.0 - b_p * sx_p) / s_p
        a_n = (1.0 - b_n * sx_n) / s_n
        t = (np.abs(a_p[k]) + np.abs(b_p[k] * xs)) * ep + (np.abs(a_n[k]) + np.abs(b_n[k] * xs)) * en
        T[off + flat[keep]] = t
    return T
