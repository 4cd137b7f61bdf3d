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
"""
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


if __name__ == "__main__":
    torch.set_num_threads(1)
    wa_unit()
    dct_small()
    design_small()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
