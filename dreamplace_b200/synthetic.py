"""Seeded synthetic placement designs (stand-ins for Bookshelf benchmarks).

The reference reads designs through its C++ ``place_io`` (Bookshelf/LEF/DEF);
no benchmark files exist on this machine, so designs are generated from a seed
with the shapes, sizes and distributions of the hot-path workloads:

* ``cells_10k``  - 3000x3000 die, 250 rows of height 12, 10,000 movable cells of
  width U{2..32}, 50 fixed macros with sides U[60,300], 10,200 nets of degree
  2+Geometric(0.45) truncated at 50, 128x128 bins.
* ``cells_2m``   - 2.1M movable cells of width round(exp(U[ln1,ln40])), 1,000
  macros, 2.2M nets, square die sized for 70% utilisation, 1024x1024 bins.
* ``scaled``     - the same generator at any cell count (``cells_50k``, batched designs).

Pins are numbered in net order, as the reference's Bookshelf reader numbers
them while reading the ``.nets`` file; 70% of a net's pins come from a
500-node index window, the rest uniformly from all physical nodes.  Pin
offsets are uniform inside the owning cell.

Derived quantities follow the reference's PlaceDB:
``dreamplace/PlaceDB.py:919-950`` (filler width = mean width of movable cells
between the 5th and 95th width percentile, height = row height, count =
round(max(space*t - movable_area, 0) / filler_area)), ``:820-824`` (target
density raised to the cell utilisation), ``:803`` (movable macro mask),
``:331-345`` (bin centres), and ``dreamplace/BasicPlace.py:269-364`` (initial
positions: movable cells at die centre + N(0, 0.001*die), fillers uniform).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Design:
    """Flat netlist + geometry in the reference PlaceDB's array conventions."""
    name: str
    xl: float
    yl: float
    xh: float
    yh: float
    row_height: float
    site_width: float
    num_movable_nodes: int
    num_terminals: int
    num_filler_nodes: int
    node_size_x: np.ndarray          # float32 [num_nodes]: movable | fixed | filler
    node_size_y: np.ndarray
    node_x: np.ndarray               # float32 [num_physical_nodes] (fixed entries meaningful)
    node_y: np.ndarray
    pin_offset_x: np.ndarray         # float32 [num_pins]
    pin_offset_y: np.ndarray
    pin2node_map: np.ndarray         # int32 [num_pins]
    pin2net_map: np.ndarray          # int32 [num_pins]
    flat_net2pin_map: np.ndarray     # int32 [num_pins]
    flat_net2pin_start_map: np.ndarray  # int32 [num_nets+1]
    flat_node2pin_map: np.ndarray    # int32 [num_pins]
    flat_node2pin_start_map: np.ndarray  # int32 [num_physical_nodes+1]
    net_weights: np.ndarray          # float32 [num_nets]
    num_bins_x: int
    num_bins_y: int
    target_density: float
    total_movable_node_area: float
    total_fixed_node_area: float
    total_space_area: float
    movable_macro_mask: np.ndarray   # bool [num_movable_nodes]
    seed: int
    extra: dict = field(default_factory=dict)

    @property
    def num_physical_nodes(self):
        return self.num_movable_nodes + self.num_terminals

    @property
    def num_nodes(self):
        return self.num_physical_nodes + self.num_filler_nodes

    @property
    def num_pins(self):
        return int(self.pin2node_map.shape[0])

    @property
    def num_nets(self):
        return int(self.flat_net2pin_start_map.shape[0] - 1)

    @property
    def width(self):
        return self.xh - self.xl

    @property
    def height(self):
        return self.yh - self.yl

    @property
    def area(self):
        return self.width * self.height

    @property
    def bin_size_x(self):
        return (self.xh - self.xl) / self.num_bins_x

    @property
    def bin_size_y(self):
        return (self.yh - self.yl) / self.num_bins_y

    def bin_centers(self, l, h, bin_size):
        """Bin centres as ``dreamplace/PlaceDB.py:331-345`` computes them."""
        num_bins = int(np.ceil((h - l) / bin_size))
        centers = np.zeros(num_bins, dtype=np.float32)
        for i in range(num_bins):
            bl = l + i * bin_size
            bh = min(bl + bin_size, h)
            centers[i] = (bl + bh) / 2
        return centers

    def initial_positions(self, seed=1000):
        """Initial ``pos`` = [x(n), y(n)] as ``dreamplace/BasicPlace.py:269-364``."""
        rng = np.random.RandomState(seed)
        n = self.num_nodes
        pos = np.zeros(2 * n, dtype=np.float32)
        pos[: self.num_physical_nodes] = self.node_x
        pos[n: n + self.num_physical_nodes] = self.node_y
        m = self.num_movable_nodes
        pos[:m] = rng.normal(loc=(self.xl + self.xh) / 2, scale=(self.xh - self.xl) * 0.001, size=m)
        pos[n: n + m] = rng.normal(loc=(self.yl + self.yh) / 2, scale=(self.yh - self.yl) * 0.001, size=m)
        if self.num_filler_nodes:
            f = self.num_filler_nodes
            pos[self.num_physical_nodes: n] = rng.uniform(
                low=self.xl, high=self.xh - self.node_size_x[-f], size=f)
            pos[n + self.num_physical_nodes:] = rng.uniform(
                low=self.yl, high=self.yh - self.node_size_y[-f], size=f)
        return pos


def _place_macros(rng, num, lo, hi, xl, yl, xh, yh, row_height, max_tries=200000):
    """Rejection-sample non-overlapping fixed macros inside the die."""
    sizes_x = rng.randint(lo, hi + 1, size=num).astype(np.float64)
    sizes_y = rng.randint(lo, hi + 1, size=num).astype(np.float64)
    xs = np.zeros(num)
    ys = np.zeros(num)
    # uniform grid hash for fast overlap tests
    cell = float(hi)
    grid = {}
    placed = 0
    tries = 0
    while placed < num:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place macros without overlap")
        w, h = sizes_x[placed], sizes_y[placed]
        x = float(rng.randint(int(xl), int(xh - w) + 1))
        y = float(rng.randint(int(yl), int(yh - h) + 1))
        gx0, gx1 = int(x // cell), int((x + w) // cell)
        gy0, gy1 = int(y // cell), int((y + h) // cell)
        ok = True
        for gx in range(gx0 - 1, gx1 + 2):
            for gy in range(gy0 - 1, gy1 + 2):
                for j in grid.get((gx, gy), ()):
                    if x < xs[j] + sizes_x[j] and xs[j] < x + w and y < ys[j] + sizes_y[j] and ys[j] < y + h:
                        ok = False
                        break
                if not ok:
                    break
            if not ok:
                break
        if not ok:
            continue
        xs[placed], ys[placed] = x, y
        for gx in range(gx0, gx1 + 1):
            for gy in range(gy0, gy1 + 1):
                grid.setdefault((gx, gy), []).append(placed)
        placed += 1
    return xs, ys, sizes_x, sizes_y


def _make_nets(rng, num_nets, num_physical, window=500, local_frac=0.7, p=0.45, max_degree=50):
    """Nets of degree 2+Geometric(p) (failures), truncated at max_degree."""
    deg = 2 + (rng.geometric(p, size=num_nets) - 1)
    deg = np.minimum(deg, max_degree).astype(np.int64)
    start = np.zeros(num_nets + 1, dtype=np.int64)
    np.cumsum(deg, out=start[1:])
    P = int(start[-1])
    net_of_pin = np.repeat(np.arange(num_nets, dtype=np.int64), deg)
    c = rng.randint(0, max(num_physical - window, 0) + 1, size=num_nets)
    local = rng.random_sample(P) < local_frac
    w = min(window, num_physical)
    node_local = c[net_of_pin] + rng.randint(0, w, size=P)
    node_any = rng.randint(0, num_physical, size=P)
    pin2node = np.where(local, node_local, node_any).astype(np.int32)
    return start.astype(np.int32), net_of_pin.astype(np.int32), pin2node


def _finish(name, seed, xl, yl, xh, yh, row_height, mov_w, mov_h, mac_x, mac_y, mac_w, mac_h,
            num_nets, num_bins, target_density, rng):
    nphys = mov_w.shape[0] + mac_w.shape[0]
    size_x = np.concatenate([mov_w, mac_w]).astype(np.float32)
    size_y = np.concatenate([mov_h, mac_h]).astype(np.float32)
    start, net_of_pin, pin2node = _make_nets(rng, num_nets, nphys)
    P = pin2node.shape[0]
    off_x = (rng.random_sample(P) * size_x[pin2node]).astype(np.float32)
    off_y = (rng.random_sample(P) * size_y[pin2node]).astype(np.float32)
    d = _finish_from_arrays(name, xl, yl, xh, yh, row_height, mov_w, mov_h, mac_x, mac_y, mac_w, mac_h, pin2node,
                            net_of_pin, start, off_x, off_y, np.ones(num_nets, dtype=np.float32), num_bins,
                            target_density)
    d.seed = seed
    return d


def _finish_from_arrays(name, xl, yl, xh, yh, row_height, mov_w, mov_h, mac_x, mac_y, mac_w, mac_h, pin2node,
                        net_of_pin, start, off_x, off_y, net_weights, num_bins, target_density):
    """Design from netlist arrays (pins in net order): node/pin CSR maps, areas,
    utilisation, target density, movable macros and fillers as the reference's
    PlaceDB derives them."""
    m = mov_w.shape[0]
    f_num = mac_w.shape[0]
    nphys = m + f_num
    size_x = np.concatenate([mov_w, mac_w]).astype(np.float32)
    size_y = np.concatenate([mov_h, mac_h]).astype(np.float32)
    node_x = np.zeros(nphys, dtype=np.float32)
    node_y = np.zeros(nphys, dtype=np.float32)
    node_x[m:] = mac_x
    node_y[m:] = mac_y
    P = pin2node.shape[0]
    num_nets = start.shape[0] - 1
    flat_net2pin = np.arange(P, dtype=np.int32)
    order = np.argsort(pin2node, kind="stable").astype(np.int32)
    counts = np.bincount(pin2node, minlength=nphys)
    node_start = np.zeros(nphys + 1, dtype=np.int32)
    np.cumsum(counts, out=node_start[1:])

    area = (xh - xl) * (yh - yl)
    total_movable_node_area = float(np.sum(mov_w.astype(np.float64) * mov_h))
    fx = np.maximum(np.minimum(mac_x + mac_w, xh) - np.maximum(mac_x, xl), 0.0)
    fy = np.maximum(np.minimum(mac_y + mac_h, yh) - np.maximum(mac_y, yl), 0.0)
    total_fixed_node_area = float(np.sum(fx * fy))
    # rows cover the whole die; macros never overlap each other
    total_space_area = area - total_fixed_node_area

    mean_area = total_movable_node_area / m
    mov_area = mov_w.astype(np.float64) * mov_h
    movable_macro_mask = (mov_area > mean_area * 10) & (mov_h > row_height * 2)
    total_movable_macro_area = float(mov_area[movable_macro_mask].sum())
    total_movable_cell_area = total_movable_node_area - total_movable_macro_area
    total_cell_space_area = total_space_area - total_movable_macro_area
    cell_utilization = total_movable_cell_area / total_cell_space_area
    target_density = max(target_density, min(cell_utilization, 1.0))

    order_w = np.argsort(size_x[:m], kind="stable")
    lb, ub = int(m * 0.05), int(m * 0.95)
    filler_w = 0.0 if lb >= ub else float(np.mean(size_x[order_w[lb:ub]]))
    filler_h = row_height
    total_filler_area = max(total_cell_space_area * target_density - total_movable_cell_area, 0.0)
    n_fill = 0 if filler_w * filler_h == 0 else int(round(total_filler_area / (filler_w * filler_h)))
    size_x = np.concatenate([size_x, np.full(n_fill, filler_w, dtype=np.float32)])
    size_y = np.concatenate([size_y, np.full(n_fill, filler_h, dtype=np.float32)])

    return Design(
        name=name, xl=float(xl), yl=float(yl), xh=float(xh), yh=float(yh),
        row_height=float(row_height), site_width=1.0,
        num_movable_nodes=m, num_terminals=f_num, num_filler_nodes=n_fill,
        node_size_x=size_x, node_size_y=size_y, node_x=node_x, node_y=node_y,
        pin_offset_x=np.asarray(off_x, np.float32), pin_offset_y=np.asarray(off_y, np.float32),
        pin2node_map=np.asarray(pin2node, np.int32), pin2net_map=np.asarray(net_of_pin, np.int32),
        flat_net2pin_map=flat_net2pin, flat_net2pin_start_map=np.asarray(start, np.int32),
        flat_node2pin_map=order, flat_node2pin_start_map=node_start,
        net_weights=np.asarray(net_weights, np.float32),
        num_bins_x=num_bins, num_bins_y=num_bins, target_density=float(target_density),
        total_movable_node_area=total_movable_node_area,
        total_fixed_node_area=total_fixed_node_area, total_space_area=total_space_area,
        movable_macro_mask=movable_macro_mask, seed=0,
        extra={"filler_size": (filler_w, filler_h), "cell_utilization": cell_utilization})


def cells_10k(seed=1):
    """The CPU-runnable parity design (10k cells, 128x128 bins)."""
    rng = np.random.RandomState(seed)
    xl, yl, xh, yh, rh = 0.0, 0.0, 3000.0, 3000.0, 12.0
    m = 10000
    mov_w = rng.randint(2, 33, size=m).astype(np.float32)
    mov_h = np.full(m, rh, dtype=np.float32)
    mx, my, mw, mh = _place_macros(rng, 50, 60, 300, xl, yl, xh, yh, rh)
    return _finish("cells10k", seed, xl, yl, xh, yh, rh, mov_w, mov_h, mx, my, mw, mh,
                   10200, 128, 1.0, rng)


def scaled(num_movable, num_nets=None, num_macros=None, num_bins=None, seed=1, utilization=0.7,
           name=None):
    """The large-design generator: log-uniform widths 1-40 sites, square die at
    ``utilization``, macros with sides U[60,300]."""
    rng = np.random.RandomState(seed)
    m = int(num_movable)
    if num_nets is None:
        num_nets = int(round(m * 2.2 / 2.1))
    if num_macros is None:
        num_macros = max(int(round(m * 1000 / 2.1e6)), 1)
    rh = 12.0
    mov_w = np.maximum(np.round(np.exp(rng.uniform(np.log(1.0), np.log(40.0), size=m))), 1.0).astype(np.float32)
    mov_h = np.full(m, rh, dtype=np.float32)
    mac_w = rng.randint(60, 301, size=num_macros).astype(np.float64)
    mac_h = rng.randint(60, 301, size=num_macros).astype(np.float64)
    mov_area = float(np.sum(mov_w.astype(np.float64) * rh))
    mac_area = float(np.sum(mac_w * mac_h))
    side = math.sqrt(mov_area / utilization + mac_area)
    side = math.ceil(side / rh) * rh
    # re-sample macro positions with the sampled sizes
    xs = np.zeros(num_macros)
    ys = np.zeros(num_macros)
    cell = 300.0
    grid = {}
    placed = 0
    tries = 0
    while placed < num_macros:
        tries += 1
        if tries > 100 * num_macros + 100000:
            raise RuntimeError("macro placement failed")
        w, h = mac_w[placed], mac_h[placed]
        x = float(rng.randint(0, int(side - w) + 1))
        y = float(rng.randint(0, int(side - h) + 1))
        gx0, gx1 = int(x // cell), int((x + w) // cell)
        gy0, gy1 = int(y // cell), int((y + h) // cell)
        ok = True
        for gx in range(gx0 - 1, gx1 + 2):
            for gy in range(gy0 - 1, gy1 + 2):
                for j in grid.get((gx, gy), ()):
                    if x < xs[j] + mac_w[j] and xs[j] < x + w and y < ys[j] + mac_h[j] and ys[j] < y + h:
                        ok = False
                        break
                if not ok:
                    break
            if not ok:
                break
        if not ok:
            continue
        xs[placed], ys[placed] = x, y
        for gx in range(gx0, gx1 + 1):
            for gy in range(gy0, gy1 + 1):
                grid.setdefault((gx, gy), []).append(placed)
        placed += 1
    if num_bins is None:
        nb = 2 ** int(round(math.log2(math.sqrt(m))))
        num_bins = int(min(max(nb, 64), 512))
    return _finish(name or f"synthetic_{m}", seed, 0.0, 0.0, side, side, rh, mov_w, mov_h,
                   xs, ys, mac_w, mac_h, num_nets, num_bins, 1.0, rng)


def cells_2m(seed=1):
    """The op-level / full-GP scale design: 2.1M cells, 2.2M nets, 1024x1024 bins."""
    return scaled(2_100_000, num_nets=2_200_000, num_macros=1000, num_bins=1024, seed=seed,
                  name="cells2100k")


def cells_50k(seed=1):
    """50k cells at 256x256 bins (finite-difference check design)."""
    return scaled(50_000, num_bins=256, seed=seed, name="cells50k")

