"""Generates tests/golden/*.npz from the reference's own CPU ops.

Run in a container that has the reference checkout (it builds the reference
CPU extensions into oracle/_ref first if they are missing):

    python oracle/build_ref.py && python tests/golden/make_golden.py

Fixtures (all float32 unless noted):

* ``wa_unit.npz``  -- the 5-pin / 2-net case of the reference's
  unittest/ops/weighted_average_wirelength_unittest.py (gamma 0.5, net weights
  [1, 2]) through weighted_average_wirelength_cpp_merged forward + backward.
* ``dct_small.npz`` -- a seeded 16 x 32 map through dct2_fft2_cpp's four transforms.
* ``design_small.npz`` -- a seeded 3,000-cell synthetic design at 64 x 64 bins with
  spread positions through electric_potential_cpp (density_map fp32 and
  deterministic, fixed_density_map, electric_force from the reference's own
  field maps), weighted_average_wirelength_cpp_merged, hpwl_cpp, pin_pos_cpp.
* ``ep_unit.npz`` -- the case of the reference's
  unittest/ops/electric_potential_unittest.py (1 movable + 83 fixed cells,
  1024 x 1024 bins; its arrays are read from that file with ``ast``) in
  float32: fixed and density maps, energy, force, and the field maps in a
  window around the movable cell.
* ``ep_options.npz`` -- the 3,000-cell design through the reference
  module's options (movable-macro mask at target density 0.8, padding 2,
  overflow mode), composed from electric_potential_cpp and dct2_fft2_cpp.
* ``dct_unit.npz`` -- the 4 x 8 inputs of the reference's
  unittest/ops/dct_unittest.py (seed 10) through dct2_fft2_cpp.
* ``wa_edge.npz`` -- a netlist of edge-case nets (degree 1, full and partial
  lane groups of degrees 2..8, degrees up to 300, coincident pins, exp
  underflow, masked nets, net weights) through pin_pos_cpp,
  weighted_average_wirelength_cpp_merged and hpwl_cpp.

``python tests/golden/make_golden.py [fixture ...]`` regenerates the named
fixtures (default: all).  The reference checkout is read from
``$DREAMPLACE_REFERENCE`` (default /root/reference).
"""
import ast
import math
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from dreamplace_b200 import synthetic  # noqa: E402


def need(name):
    m = oracle.load_ref(name)
    if m is None:
        raise SystemExit("reference op %s not built; run python oracle/build_ref.py" % name)
    return m


def t(a, dtype=None):
    x = torch.from_numpy(np.ascontiguousarray(a))
    return x if dtype is None else x.to(dtype)


def wa_unit():
    wa = need("weighted_average_wirelength_cpp_merged")
    pin_pos = np.array([[0.0, 0.0], [1.0, 2.0], [1.5, 0.2], [0.5, 3.1], [0.6, 1.1]], dtype=np.float32)
    nets = [[0, 4], [1, 2, 3]]
    flat = np.array([p for n in nets for p in n], np.int32)
    start = np.array([0, 2, 5], np.int32)
    pin2net = np.zeros(5, np.int32)
    for i, n in enumerate(nets):
        pin2net[n] = i
    weights = np.array([1, 2], np.float32)
    mask = np.ones(2, np.uint8)
    gamma = 0.5
    pos = np.concatenate([pin_pos[:, 0], pin_pos[:, 1]]).astype(np.float32)
    inv_gamma = torch.tensor([1.0 / gamma], dtype=torch.float32)
    wl, gi = wa.forward(t(pos), t(flat), t(start), t(pin2net), t(weights), t(mask), inv_gamma)
    grad = wa.backward(torch.ones(1), t(pos), gi.clone(), t(flat), t(start), t(pin2net), t(weights), t(mask),
                       inv_gamma)
    np.savez_compressed(os.path.join(HERE, "wa_unit.npz"), pos=pos, flat_netpin=flat, netpin_start=start,
                        pin2net=pin2net, net_weights=weights, net_mask=mask, gamma=np.float32(gamma),
                        wl=np.float32(wl.item()), grad_intermediate=gi.numpy(), grad=grad.numpy())


def dct_small():
    d = need("dct2_fft2_cpp")
    rng = np.random.RandomState(10)
    M, N = 16, 32
    x = rng.uniform(-1, 1, size=(M, N)).astype(np.float32)
    res = {"x": x}
    for name in ("dct2_fft2", "idct2_fft2", "idct_idxst", "idxst_idct"):
        expkM = oracle_expk(M)
        expkN = oracle_expk(N)
        out = torch.empty(M, N)
        buf = torch.empty(M, N // 2 + 1, 2)
        getattr(d, name)(t(x), expkM, expkN, out, buf, 1)
        res[name] = out.numpy().copy()
    np.savez_compressed(os.path.join(HERE, "dct_small.npz"), **res)


def oracle_expk(n):
    u = torch.arange(n, dtype=torch.float32).mul_(np.pi / (2 * n))
    return torch.stack([u.cos(), -u.sin()], dim=-1).contiguous()


def design_small():
    ep = need("electric_potential_cpp")
    dct = need("dct2_fft2_cpp")
    wa = need("weighted_average_wirelength_cpp_merged")
    hp = need("hpwl_cpp")
    pp = need("pin_pos_cpp")
    d = synthetic.scaled(3000, num_bins=64, seed=7, name="golden_small")
    rng = np.random.RandomState(11)
    n = d.num_nodes
    pos = d.initial_positions(seed=12)
    m = d.num_movable_nodes
    pos[:m] = rng.uniform(d.xl, d.xh - d.node_size_x[:m], size=m)
    pos[n:n + m] = rng.uniform(d.yl, d.yh - d.node_size_y[:m], size=m)
    pos = pos.astype(np.float32)
    M = N = d.num_bins_x
    bsx, bsy = d.bin_size_x, d.bin_size_y
    bcx = d.bin_centers(d.xl, d.xh, bsx)
    bcy = d.bin_centers(d.yl, d.yh, bsy)
    sx = t(d.node_size_x)
    sy = t(d.node_size_y)
    sxc = sx.clamp(min=bsx * math.sqrt(2))
    syc = sy.clamp(min=bsy * math.sqrt(2))
    ox = (sx - sxc).mul(0.5)
    oy = (sy - syc).mul(0.5)
    ratio = sx * sy / (sxc * syc)
    tpos = t(pos)
    nt, nf = d.num_terminals, d.num_filler_nodes
    res = dict(pos=pos, M=M, N=N)
    for det in (0, 1):
        fixed = ep.fixed_density_map(tpos, sx, sy, t(bcx), t(bcy), d.xl, d.yl, d.xh, d.yh, bsx, bsy, m, nt, M, N,
                                     0, 0, det)
        res["fixed_map_det%d" % det] = fixed.numpy().copy()
        init = fixed.mul(d.target_density)
        dm = ep.density_map(tpos, sxc, syc, ox, oy, ratio, t(bcx), t(bcy), init, d.target_density, d.xl, d.yl,
                            d.xh, d.yh, bsx, bsy, m, nf, 0, M, N, 0, 0, 0, 0, det)
        res["density_map_det%d" % det] = dm.numpy().copy()
    # reference field maps (FFT path) for the deterministic density map, then the force
    rho = t(res["density_map_det1"]).view(M, N).clone().mul_(1.0 / (bsx * bsy))
    expkM, expkN = oracle_expk(M), oracle_expk(N)
    buf = torch.empty(M, N // 2 + 1, 2)
    auv = torch.empty(M, N)
    dct.dct2_fft2(rho, expkM, expkN, auv, buf, 1)
    wu = torch.arange(M, dtype=torch.float32).mul(2 * np.pi / M).view([M, 1])
    wv = torch.arange(N, dtype=torch.float32).mul(2 * np.pi / N).view([1, N]).mul_(bsx / bsy)
    w2 = wu.pow(2) + wv.pow(2)
    w2[0, 0] = 1.0
    inv = 1.0 / w2
    inv[0, 0] = 0.0
    ex = torch.empty(M, N)
    ey = torch.empty(M, N)
    dct.idxst_idct(auv.mul(wu.mul(inv).mul_(0.5)), expkM, expkN, ex, buf, 1)
    dct.idct_idxst(auv.mul(wv.mul(inv).mul_(0.5)), expkM, expkN, ey, buf, 1)
    phi = torch.empty(M, N)
    dct.idct2_fft2(auv.mul(inv), expkM, expkN, phi, buf, 1)
    res.update(field_x=ex.numpy().copy(), field_y=ey.numpy().copy(), energy=np.float32((phi * rho).sum().item()))
    grad = torch.ones(1)
    force = ep.electric_force(grad, M, N, 0, 0, 0, 0, ex.view(-1), ey.view(-1), tpos, sxc, syc, ox, oy, ratio,
                              t(bcx), t(bcy), d.xl, d.yl, d.xh, d.yh, bsx, bsy, m, nf)
    res["force"] = (-force).numpy().copy()
    # pins / nets
    p2n = t(d.pin2node_map.astype(np.int64))
    pin = pp.forward(tpos, t(d.pin_offset_x), t(d.pin_offset_y), p2n, t(d.flat_node2pin_map),
                     t(d.flat_node2pin_start_map))
    res["pin_pos"] = pin.numpy().copy()
    rg = np.random.RandomState(13).uniform(-1, 1, size=2 * d.num_pins).astype(np.float32)
    res["pin_grad_in"] = rg
    res["pin_pos_backward"] = pp.backward(t(rg), tpos, t(d.pin_offset_x), t(d.pin_offset_y), p2n,
                                          t(d.flat_node2pin_map), t(d.flat_node2pin_start_map),
                                          d.num_physical_nodes).numpy().copy()
    deg = np.diff(d.flat_net2pin_start_map)
    mask = ((deg >= 2) & (deg < 100)).astype(np.uint8)
    res["net_mask"] = mask
    gamma = 4.0 * (bsx + bsy)
    res["inv_gamma"] = np.float32(1.0 / gamma)
    inv_gamma = torch.tensor([1.0 / gamma], dtype=torch.float32)
    wl, gi = wa.forward(pin, t(d.flat_net2pin_map), t(d.flat_net2pin_start_map), t(d.pin2net_map),
                        t(d.net_weights), t(mask), inv_gamma)
    res["wa_wl"] = np.float32(wl.item())
    res["wa_grad_intermediate"] = gi.numpy().copy()
    res["hpwl"] = np.float32(hp.forward(pin, t(d.flat_net2pin_map), t(d.flat_net2pin_start_map),
                                        t(d.net_weights), t((deg >= 2).astype(np.uint8))).item())
    np.savez_compressed(os.path.join(HERE, "design_small.npz"), **res)


# ---------------------------------------------------------------- reference unit-test cases
REF = os.environ.get("DREAMPLACE_REFERENCE", "/root/reference")


def reference_test_literals(relpath, func):
    """The literal assignments (numbers, and ``np.array([...])`` lists with an
    optional ``.astype``) of one test function of a reference unit-test file,
    read with ``ast`` when the fixture is generated."""
    tree = ast.parse(open(os.path.join(REF, relpath)).read())
    fn = next(n for n in ast.walk(tree) if isinstance(n, ast.FunctionDef) and n.name == func)
    out = {}
    for st in fn.body:
        if not (isinstance(st, ast.Assign) and len(st.targets) == 1 and isinstance(st.targets[0], ast.Name)):
            continue
        v = st.value
        if isinstance(v, ast.Call) and isinstance(v.func, ast.Attribute) and v.func.attr == "astype":
            v = v.func.value
        if isinstance(v, ast.Call) and isinstance(v.func, ast.Attribute) and v.func.attr == "array" and v.args:
            v = v.args[0]
        try:
            out[st.targets[0].id] = ast.literal_eval(v)
        except ValueError:
            pass
    return out


def bin_centers(lo, hi, size, n):
    c = np.zeros(n, np.float32)
    for i in range(n):
        bl = lo + i * size
        c[i] = (bl + min(bl + size, hi)) / 2
    return c


def ep_unit():
    """The reference's electric-potential unit test case
    (unittest/ops/electric_potential_unittest.py, test_densityOverflowRandom):
    one movable cell and 83 fixed cells (one of them as wide as the die) on a
    16728 x 11424 die starting at y = 6, 1024 x 1024 bins, target density 0.7,
    here in float32.  Field maps are kept only in a window around the movable
    cell (the bins its force reads)."""
    ep = need("electric_potential_cpp")
    dct = need("dct2_fft2_cpp")
    a = reference_test_literals("unittest/ops/electric_potential_unittest.py", "test_densityOverflowRandom")
    xx, yy = np.array(a["xx"], np.float32), np.array(a["yy"], np.float32)
    sxn, syn = np.array(a["node_size_x"], np.float32), np.array(a["node_size_y"], np.float32)
    n, m = len(xx), int(a["num_movable_nodes"])
    nt, nf = n - m, 0
    xl, yl, xh, yh = (float(a[k]) for k in ("xl", "yl", "xh", "yh"))
    M, N = int(a["num_bins_x"]), int(a["num_bins_y"])
    target = float(a["target_density"])
    bsx, bsy = (xh - xl) / M, (yh - yl) / N
    bcx, bcy = bin_centers(xl, xh, bsx, M), bin_centers(yl, yh, bsy, N)
    pos = np.concatenate([xx, yy]).astype(np.float32)
    sx, sy = t(sxn), t(syn)
    sxc = sx.clamp(min=bsx * math.sqrt(2))
    syc = sy.clamp(min=bsy * math.sqrt(2))
    ox = (sx - sxc).mul(0.5)
    oy = (sy - syc).mul(0.5)
    ratio = sx * sy / (sxc * syc)
    tpos = t(pos)
    res = dict(pos=pos, node_size_x=sxn, node_size_y=syn, num_movable=m, num_terminals=nt,
               geometry=np.array([xl, yl, xh, yh], np.float64), bins=np.array([M, N]), target_density=target)
    for det in (0, 1):
        fixed = ep.fixed_density_map(tpos, sx, sy, t(bcx), t(bcy), xl, yl, xh, yh, bsx, bsy, m, nt, M, N, 0, 0, det)
        res["fixed_map_det%d" % det] = fixed.numpy().copy()
        dm = ep.density_map(tpos, sxc, syc, ox, oy, ratio, t(bcx), t(bcy), fixed.mul(target), target, xl, yl, xh,
                            yh, bsx, bsy, m, nf, 0, M, N, 0, 0, 0, 0, det)
        res["density_map_det%d" % det] = dm.numpy().copy()
    rho = t(res["density_map_det1"]).view(M, N).clone().mul_(1.0 / (bsx * bsy))
    expkM, expkN = oracle_expk(M), oracle_expk(N)
    buf = torch.empty(M, N // 2 + 1, 2)
    auv = torch.empty(M, N)
    dct.dct2_fft2(rho, expkM, expkN, auv, buf, 1)
    wu = torch.arange(M, dtype=torch.float32).mul(2 * np.pi / M).view([M, 1])
    wv = torch.arange(N, dtype=torch.float32).mul(2 * np.pi / N).view([1, N]).mul_(bsx / bsy)
    w2 = wu.pow(2) + wv.pow(2)
    w2[0, 0] = 1.0
    inv = 1.0 / w2
    inv[0, 0] = 0.0
    ex, ey, phi = torch.empty(M, N), torch.empty(M, N), torch.empty(M, N)
    dct.idxst_idct(auv.mul(wu.mul(inv).mul_(0.5)), expkM, expkN, ex, buf, 1)
    dct.idct_idxst(auv.mul(wv.mul(inv).mul_(0.5)), expkM, expkN, ey, buf, 1)
    dct.idct2_fft2(auv.mul(inv), expkM, expkN, phi, buf, 1)
    res["energy"] = np.float32((phi * rho).sum().item())
    force = ep.electric_force(torch.ones(1), M, N, 0, 0, 0, 0, ex.view(-1), ey.view(-1), tpos, sxc, syc, ox, oy,
                              ratio, t(bcx), t(bcy), xl, yl, xh, yh, bsx, bsy, m, nf)
    res["force"] = (-force).numpy().copy()
    # window of bins around the movable cells' stretched footprints, 4 bins of margin
    xs = pos[:m] + ox.numpy()[:m]
    ys = pos[n:n + m] + oy.numpy()[:m]
    k0 = max(int(np.floor((xs.min() - xl) / bsx)) - 4, 0)
    k1 = min(int(np.ceil((xs.max() + sxc.numpy()[:m].max() - xl) / bsx)) + 4, M)
    h0 = max(int(np.floor((ys.min() - yl) / bsy)) - 4, 0)
    h1 = min(int(np.ceil((ys.max() + syc.numpy()[:m].max() - yl) / bsy)) + 4, N)
    res["field_window"] = np.array([k0, k1, h0, h1])
    res["field_x_window"] = ex[k0:k1, h0:h1].numpy().copy()
    res["field_y_window"] = ey[k0:k1, h0:h1].numpy().copy()
    np.savez_compressed(os.path.join(HERE, "ep_unit.npz"), **res)


def dct_unit():
    """The reference's 2-D transform unit-test inputs (unittest/ops/dct_unittest.py
    test_dct2Random and the inverse tests: seed 10, 4 x 8; U[0, 10) for DCT2,
    integers 0..9 for the inverse transforms), in float32, through
    dct2_fft2_cpp's four transforms."""
    d = need("dct2_fft2_cpp")
    M, N = 4, 8
    torch.manual_seed(10)
    x = torch.empty(M, N, dtype=torch.float32).uniform_(0, 10.0)
    torch.manual_seed(10)
    xi = torch.empty(M, N, dtype=torch.int32).random_(0, 10).float()
    res = {"x": x.numpy().copy(), "x_int": xi.numpy().copy()}
    expkM, expkN = oracle_expk(M), oracle_expk(N)
    for name in ("dct2_fft2", "idct2_fft2", "idct_idxst", "idxst_idct"):
        src = x if name == "dct2_fft2" else xi
        out = torch.empty(M, N)
        buf = torch.empty(M, N // 2 + 1, 2)
        getattr(d, name)(src.contiguous(), expkM, expkN, out, buf, 1)
        res[name] = out.numpy().copy()
    np.savez_compressed(os.path.join(HERE, "dct_unit.npz"), **res)


def wa_edge():
    """Nets the synthetic designs do not have: degree 1 (unmasked, as the
    reference's mask keeps them), full and partial groups of every degree
    2..8, degrees 9..300, all pins of a net on one point, a net spread far
    beyond gamma (exp underflow), masked nets; random net weights.  Pins sit
    on shared nodes with offsets; the reference ops see the pin positions."""
    wa = need("weighted_average_wirelength_cpp_merged")
    hp = need("hpwl_cpp")
    pp = need("pin_pos_cpp")
    rng = np.random.RandomState(21)
    degrees = [d for d in range(1, 9) for _ in range(37)] + [9, 12, 16, 31, 32, 33, 40, 64, 65, 150, 300]
    degrees = list(rng.permutation(degrees)) + [5, 9]  # the last two: coincident and far-spread
    E = len(degrees)
    P = int(sum(degrees))
    n = P // 3
    pin2node = rng.randint(0, n, size=P).astype(np.int32)
    offx = rng.uniform(0, 4, size=P).astype(np.float32)
    offy = rng.uniform(0, 4, size=P).astype(np.float32)
    node_x = rng.uniform(0, 1000, size=n).astype(np.float32)
    node_y = rng.uniform(0, 1000, size=n).astype(np.float32)
    flat = rng.permutation(P).astype(np.int32)  # pins of a net are not consecutive ids
    start = np.concatenate([[0], np.cumsum(degrees)]).astype(np.int32)
    # coincident net: every pin on one node, zero offsets
    cpins = flat[start[E - 2]:start[E - 1]]
    pin2node[cpins] = pin2node[cpins[0]]
    offx[cpins] = 0
    offy[cpins] = 0
    # far-spread net: its own nodes, x from 0 to 1e5
    fpins = flat[start[E - 1]:start[E]]
    fnodes = np.arange(n - len(fpins), n)
    pin2node[fpins] = fnodes
    node_x[fnodes] = np.linspace(0, 1e5, len(fpins)).astype(np.float32)
    pin2net = np.zeros(P, np.int32)
    for e in range(E):
        pin2net[flat[start[e]:start[e + 1]]] = e
    mask = np.ones(E, np.uint8)
    mask[::7] = 0
    mask[E - 2:] = 1
    weights = rng.uniform(0.5, 2.0, size=E).astype(np.float32)
    pos = np.concatenate([node_x, node_y]).astype(np.float32)
    order = np.argsort(pin2node, kind="stable").astype(np.int32)  # node -> pin CSR
    node_start = np.concatenate([[0], np.cumsum(np.bincount(pin2node, minlength=n))]).astype(np.int32)
    pin = pp.forward(t(pos), t(offx), t(offy), t(pin2node.astype(np.int64)), t(order), t(node_start))
    gamma = 8.0
    inv_gamma = torch.tensor([1.0 / gamma], dtype=torch.float32)
    wl, gi = wa.forward(pin, t(flat), t(start), t(pin2net), t(weights), t(mask), inv_gamma)
    grad = wa.backward(torch.ones(1), pin, gi.clone(), t(flat), t(start), t(pin2net), t(weights), t(mask),
                       inv_gamma)
    hmask = (np.diff(start) >= 2).astype(np.uint8)
    h = hp.forward(pin, t(flat), t(start), t(weights), t(hmask))
    np.savez_compressed(os.path.join(HERE, "wa_edge.npz"), pos=pos, pin2node=pin2node, pin_offset_x=offx,
                        pin_offset_y=offy, flat_node2pin=order, node_start=node_start, flat_netpin=flat,
                        netpin_start=start, pin2net=pin2net, net_mask=mask, net_weights=weights,
                        hpwl_mask=hmask, gamma=np.float32(gamma), pin_pos=pin.numpy().copy(),
                        wl=np.float32(wl.item()), grad_intermediate=gi.numpy().copy(), grad=grad.numpy().copy(),
                        hpwl=np.float32(h.item()))


def ep_options():
    """The seeded 3,000-cell design through the reference module's options,
    composed from the reference ops as dreamplace/ops/electric_potential/
    electric_overflow.py:162-278 and electric_potential.py:52-217 do:
    target density 0.8 with a movable-macro mask (ratio := target density for
    the 40 largest movable cells), padding 2 (padding bins filled with
    target x bin area), deterministic maps; the energy, the force, and the
    overflow mode (movable cells only)."""
    ep = need("electric_potential_cpp")
    dct = need("dct2_fft2_cpp")
    d = synthetic.scaled(3000, num_bins=64, seed=7, name="golden_small")
    pos = np.load(os.path.join(HERE, "design_small.npz"))["pos"]
    n, m, nt, nf = d.num_nodes, d.num_movable_nodes, d.num_terminals, d.num_filler_nodes
    M = N = d.num_bins_x
    bsx, bsy = d.bin_size_x, d.bin_size_y
    target, padding = 0.8, 2
    bcx = d.bin_centers(d.xl, d.xh, bsx)
    bcy = d.bin_centers(d.yl, d.yh, bsy)
    sx, sy = t(d.node_size_x), t(d.node_size_y)
    sxc = sx.clamp(min=bsx * math.sqrt(2))
    syc = sy.clamp(min=bsy * math.sqrt(2))
    ox = (sx - sxc).mul(0.5)
    oy = (sy - syc).mul(0.5)
    ratio = sx * sy / (sxc * syc)
    area = d.node_size_x[:m] * d.node_size_y[:m]
    macro = np.zeros(m, bool)
    macro[np.argsort(-area, kind="stable")[:40]] = True
    ratio[:m][t(macro)] = target
    pad = torch.ones(M, N, dtype=torch.bool)
    pad[padding:M - padding, padding:N - padding] = False
    tpos = t(pos)
    init = ep.fixed_density_map(tpos, sx, sy, t(bcx), t(bcy), d.xl, d.yl, d.xh, d.yh, bsx, bsy, m, nt, M, N, 0, 0,
                                1).mul(target)

    def dmap(num_filler):
        out = ep.density_map(tpos, sxc, syc, ox, oy, ratio, t(bcx), t(bcy), init, target, d.xl, d.yl, d.xh, d.yh,
                             bsx, bsy, m, num_filler, padding, M, N, 0, 0, 0, 0, 1).view(M, N)
        out.masked_fill_(pad, target * bsx * bsy)
        return out

    dm = dmap(nf)
    res = dict(macro_mask=macro.astype(np.uint8), target_density=target, padding=padding,
               density_map=dm.numpy().copy())
    rho = dm.clone().mul_(1.0 / (bsx * bsy))
    expkM, expkN = oracle_expk(M), oracle_expk(N)
    buf = torch.empty(M, N // 2 + 1, 2)
    auv = torch.empty(M, N)
    dct.dct2_fft2(rho, expkM, expkN, auv, buf, 1)
    wu = torch.arange(M, dtype=torch.float32).mul(2 * np.pi / M).view([M, 1])
    wv = torch.arange(N, dtype=torch.float32).mul(2 * np.pi / N).view([1, N]).mul_(bsx / bsy)
    w2 = wu.pow(2) + wv.pow(2)
    w2[0, 0] = 1.0
    inv = 1.0 / w2
    inv[0, 0] = 0.0
    ex, ey, phi = torch.empty(M, N), torch.empty(M, N), torch.empty(M, N)
    dct.idxst_idct(auv.mul(wu.mul(inv).mul_(0.5)), expkM, expkN, ex, buf, 1)
    dct.idct_idxst(auv.mul(wv.mul(inv).mul_(0.5)), expkM, expkN, ey, buf, 1)
    dct.idct2_fft2(auv.mul(inv), expkM, expkN, phi, buf, 1)
    res.update(field_x=ex.numpy().copy(), field_y=ey.numpy().copy(), energy=np.float32((phi * rho).sum().item()))
    force = ep.electric_force(torch.ones(1), M, N, 0, 0, 0, 0, ex.view(-1), ey.view(-1), tpos, sxc, syc, ox, oy,
                              ratio, t(bcx), t(bcy), d.xl, d.yl, d.xh, d.yh, bsx, bsy, m, nf)
    res["force"] = (-force).numpy().copy()
    om = dmap(0)
    bin_area = bsx * bsy
    res["overflow_map"] = om.numpy().copy()
    res["overflow"] = np.float32((om - target * bin_area).clamp_(min=0.0).sum().item())
    res["max_density"] = np.float32(om.max().item() / bin_area)
    np.savez_compressed(os.path.join(HERE, "ep_options.npz"), **res)


def _unwrap_arrays(node):
    """np.array(x, ...) / x.astype(...) -> x, recursively, so nested array
    literals (lists of index arrays) evaluate with ast.literal_eval."""
    class Strip(ast.NodeTransformer):
        def visit_Call(self, call):
            self.generic_visit(call)
            f = call.func
            if isinstance(f, ast.Attribute) and f.attr == "array" and call.args:
                return call.args[0]
            if isinstance(f, ast.Attribute) and f.attr == "astype":
                return f.value
            return call
    return Strip().visit(node)


def reference_test_values(relpath, func):
    """Like reference_test_literals, with nested np.array literals unwrapped."""
    tree = ast.parse(open(os.path.join(REF, relpath)).read())
    fn = next(n for n in ast.walk(tree) if isinstance(n, ast.FunctionDef) and n.name == func)
    out = {}
    for st in fn.body:
        if isinstance(st, ast.Assign) and len(st.targets) == 1 and isinstance(st.targets[0], ast.Name):
            try:
                out[st.targets[0].id] = ast.literal_eval(_unwrap_arrays(st.value))
            except ValueError:
                pass
    return out


def ops_unit():
    """The reference's unit-test cases of the ops beside the hot path, through
    its CPU ops: hpwl (unittest/ops/hpwl_unittest.py, test_hpwlRandom: 5 pins,
    2 weighted nets), pin_pos (unittest/ops/pin_pos_unittest.py,
    test_pin_pos_random: 2 physical nodes, 5 pins; the test flattens its 3 x 2
    position array row-major, so x = (1, 10, 2), y = (20, 3, 30)) forward and
    the backward of sum(pin_pos), and move_boundary
    (unittest/ops/move_boundary_unittest.py: 2 movable cells, one outside the
    die)."""
    hp, pp, mb = need("hpwl_cpp"), need("pin_pos_cpp"), need("move_boundary_cpp")
    res = {}
    a = reference_test_values("unittest/ops/hpwl_unittest.py", "test_hpwlRandom")
    pin = np.array(a["pin_pos"], np.float32)
    nets = a["net2pin_map"]
    flat = np.array([q for n in nets for q in n], np.int32)
    start = np.r_[0, np.cumsum([len(n) for n in nets])].astype(np.int32)
    weights = np.array(a["net_weights"], np.float32)
    mask = np.ones(len(nets), np.uint8)  # the test's mask: degree <= max degree
    pos = np.concatenate([pin[:, 0], pin[:, 1]]).astype(np.float32)
    res.update(hpwl_pin_pos=pos, hpwl_flat_netpin=flat, hpwl_netpin_start=start, hpwl_net_weights=weights,
               hpwl_net_mask=mask,
               hpwl=np.float32(hp.forward(t(pos), t(flat), t(start), t(weights), t(mask)).item()))
    a = reference_test_values("unittest/ops/pin_pos_unittest.py", "test_pin_pos_random")
    pos = np.array(a["pos"], np.float32).reshape(-1)
    node2pin = a["node2pin_map"]
    num_pins = sum(len(q) for q in node2pin)
    p2n = np.zeros(num_pins, np.int32)
    for node, pins in enumerate(node2pin):
        p2n[list(pins)] = node
    fn2p = np.array([q for pins in node2pin for q in pins], np.int32)
    nstart = np.r_[0, np.cumsum([len(q) for q in node2pin])].astype(np.int32)
    offx, offy = np.array(a["pin_offset_x"], np.float32), np.array(a["pin_offset_y"], np.float32)
    tp = t(pos)
    out = pp.forward(tp, t(offx), t(offy), t(p2n.astype(np.int64)), t(fn2p), t(nstart))
    back = pp.backward(torch.ones(2 * num_pins), tp, t(offx), t(offy), t(p2n.astype(np.int64)), t(fn2p), t(nstart),
                       len(node2pin))
    res.update(pp_pos=pos, pp_offset_x=offx, pp_offset_y=offy, pp_pin2node=p2n, pp_flat_node2pin=fn2p,
               pp_node_start=nstart, pp_num_physical=np.int32(len(node2pin)), pin_pos=out.numpy().copy(),
               pin_pos_backward=back.numpy().copy())
    a = reference_test_values("unittest/ops/move_boundary_unittest.py", "test_densityOverflowRandom")
    xx, yy = np.array(a["xx"], np.float32), np.array(a["yy"], np.float32)
    sx, sy = np.array(a["node_size_x"], np.float32), np.array(a["node_size_y"], np.float32)
    box = np.array([a["xl"], a["yl"], a["xh"], a["yh"]], np.float64)
    mpos = np.concatenate([xx, yy])
    num_movable = len(xx)  # the test's num_movable_nodes = len(xx)
    moved = mb.forward(t(mpos.copy()), t(sx), t(sy), *[float(v) for v in box], num_movable,
                       int(a["num_filler_nodes"]))
    res.update(mb_pos=mpos, mb_node_size_x=sx, mb_node_size_y=sy, mb_box=box,
               mb_num_movable=np.int32(num_movable), mb_num_filler=np.int32(a["num_filler_nodes"]),
               move_boundary=moved.numpy().copy())
    np.savez_compressed(os.path.join(HERE, "ops_unit.npz"), **res)


FIXTURES = {"wa_unit": wa_unit, "dct_small": dct_small, "design_small": design_small, "ep_unit": ep_unit,
            "dct_unit": dct_unit, "wa_edge": wa_edge, "ep_options": ep_options, "ops_unit": ops_unit}

if __name__ == "__main__":
    torch.set_num_threads(1)
    for name in sys.argv[1:] or list(FIXTURES):
        FIXTURES[name]()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
