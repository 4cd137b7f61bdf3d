"""Hand-written adjoints against fp64 central finite differences and the
reference's own backward (the 50k-cell, 256x256-bin differentiation design).

* WA wirelength: the kernel gradient (PinPos + WeightedAverageWirelength
  autograd) matches fp64 central differences of an fp64 WA model, and the
  reference CPU ops' backward (oracle/_ref) to 1e-5.
* Density: the reference's density gradient is the ePlace field force
  q_i * E_i, not the exact derivative of its own discrete energy
  sum(phi * rho): with the normalisation rho = D / bin_area the two differ by
  the constant 2 / (bin_area * bin_size) per axis, up to discretisation (the
  force averages the spectral field over the cell, the energy difference
  sees the potential at the cell edges).  The test measures that relation on
  fp64 central differences of the energy (fitted scale within 25% of 1,
  cosine similarity > 0.9).
h = 1e-3 * bin width, 256 random movable cells, x and y."""
import math

import numpy as np
import pytest
import torch

import oracle
from dreamplace_b200 import synthetic

pytestmark = pytest.mark.gpu

F64 = torch.float64


@pytest.fixture(scope="module")
def setup():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    d = synthetic.scaled(50000, num_bins=256, seed=4, name="fd50k")
    pos = d.initial_positions()
    rng = np.random.RandomState(8)
    n, m = d.num_nodes, d.num_movable_nodes
    pos[:m] = rng.uniform(d.xl + 50, d.xh - 90, size=m)
    pos[n:n + m] = rng.uniform(d.yl + 50, d.yh - 60, size=m)
    cells = rng.choice(m, size=256, replace=False)
    return d, pos.astype(np.float32), cells


def wa_fp64(d, pos, gamma, mask):
    """fp64 WA wirelength of node positions pos [2n] (torch, fp64, cuda)."""
    n = d.num_nodes
    dev = pos.device
    p2n = torch.from_numpy(d.pin2node_map.astype(np.int64)).to(dev)
    net = torch.from_numpy(d.pin2net_map.astype(np.int64)).to(dev)
    keep = torch.from_numpy(mask.astype(bool)).to(dev)[net]
    total = torch.zeros((), dtype=F64, device=dev)
    E = d.num_nets
    for axis, off in ((0, d.pin_offset_x), (1, d.pin_offset_y)):
        x = pos[axis * n:(axis + 1) * n][p2n] + torch.from_numpy(off.astype(np.float64)).to(dev)
        x = x[keep]
        nt = net[keep]
        xmax = torch.full((E,), -1e300, dtype=F64, device=dev).scatter_reduce(0, nt, x, "amax")
        xmin = torch.full((E,), 1e300, dtype=F64, device=dev).scatter_reduce(0, nt, x, "amin")
        ep = torch.exp((x - xmax[nt]) / gamma)
        en = torch.exp((xmin[nt] - x) / gamma)
        z = lambda v: torch.zeros(E, dtype=F64, device=dev).index_add_(0, nt, v)  # noqa: E731
        sp, sn, xsp, xsn = z(ep), z(en), z(x * ep), z(x * en)
        ok = sp > 0
        total = total + (xsp[ok] / sp[ok] - xsn[ok] / sn[ok]).sum()
    return total


def density_fp64(d, pos, s):
    """fp64 triangle-model density map (movable + filler) of pos [2n]."""
    sxc, syc, ox, oy, ratio = [torch.from_numpy(a.astype(np.float64)).to(pos.device) for a in s]
    n, m, nf = d.num_nodes, d.num_movable_nodes, d.num_filler_nodes
    idx = torch.cat([torch.arange(m), torch.arange(n - nf, n)]).to(pos.device)
    x = pos[:n][idx] + ox[idx]
    y = pos[n:][idx] + oy[idx]
    w, h, r = sxc[idx], syc[idx], ratio[idx]
    M, N = d.num_bins_x, d.num_bins_y
    bsx, bsy = d.bin_size_x, d.bin_size_y
    k0 = torch.floor((x - d.xl) / bsx).clamp(min=0).long()
    k1 = (torch.floor((x + w - d.xl) / bsx) + 1).clamp(max=M).long()
    h0 = torch.floor((y - d.yl) / bsy).clamp(min=0).long()
    h1 = (torch.floor((y + h - d.yl) / bsy) + 1).clamp(max=N).long()
    out = torch.zeros(M * N, dtype=F64, device=pos.device)
    for dk in range(int((k1 - k0).max())):
        k = k0 + dk
        px = torch.minimum(x + w, d.xl + (k + 1) * bsx) - torch.maximum(x, d.xl + k * bsx)
        for dh in range(int((h1 - h0).max())):
            hh = h0 + dh
            py = torch.minimum(y + h, d.yl + (hh + 1) * bsy) - torch.maximum(y, d.yl + hh * bsy)
            ok = (k < k1) & (hh < h1)
            out.index_add_(0, (k * N + hh)[ok], (px * py * r)[ok])
    return out.view(M, N)


def energy_fp64(d, dmap, init, mats):
    cM, chM, shM, cN, chN, shN, inv = mats
    M, N = dmap.shape
    rho = (dmap + init) / (d.bin_size_x * d.bin_size_y)
    a = 4.0 / (M * N) * cM @ rho @ cN.T
    phi = 4.0 * chM @ (a * inv) @ chN.T
    return (phi * rho).sum()


def test_wa_adjoint_fd_and_reference(setup):
    from dreamplace_b200.placement_ops import PinPos
    from dreamplace_b200.weighted_average_wirelength import WeightedAverageWirelength
    d, pos_np, cells = setup
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    deg = np.diff(d.flat_net2pin_start_map)
    mask = ((deg >= 2) & (deg < 100)).astype(np.uint8)
    gamma = 4.0 * (d.bin_size_x + d.bin_size_y)
    pos = t(pos_np).requires_grad_(True)
    pp = PinPos(t(d.pin_offset_x), t(d.pin_offset_y), t(d.pin2node_map), t(d.flat_node2pin_map),
                t(d.flat_node2pin_start_map), d.num_physical_nodes)
    wa = WeightedAverageWirelength(t(d.flat_net2pin_map), t(d.flat_net2pin_start_map), t(d.pin2net_map),
                                   t(d.net_weights), t(mask), t(d.pin2node_map >= d.num_movable_nodes),
                                   torch.tensor(gamma, device=dev), algorithm="merged")
    wa(pp(pos)).backward()
    grad = pos.grad.double().cpu().numpy()
    n = d.num_nodes
    p64 = t(pos_np.astype(np.float64))
    hstep = 1e-3 * d.bin_size_x
    fd = []
    for c in cells:
        for axis in (0, 1):
            i = axis * n + int(c)
            pp_, pm_ = p64.clone(), p64.clone()
            pp_[i] += hstep
            pm_[i] -= hstep
            fd.append(float(wa_fp64(d, pp_, gamma, mask) - wa_fp64(d, pm_, gamma, mask)) / (2 * hstep))
    fd = np.array(fd)
    got = np.array([grad[axis * n + int(c)] for c in cells for axis in (0, 1)])
    scale = np.max(np.abs(fd))
    assert np.max(np.abs(got - fd)) <= 2e-3 * scale, np.max(np.abs(got - fd)) / scale
    ref_wa = oracle.load_ref("weighted_average_wirelength_cpp_merged")
    ref_pp = oracle.load_ref("pin_pos_cpp")
    if ref_wa is not None and ref_pp is not None:
        c = lambda a: torch.from_numpy(np.ascontiguousarray(a))  # noqa: E731
        p2n = c(d.pin2node_map.astype(np.int64))
        pin = ref_pp.forward(c(pos_np), c(d.pin_offset_x), c(d.pin_offset_y), p2n, c(d.flat_node2pin_map),
                             c(d.flat_node2pin_start_map))
        ig = torch.tensor([1.0 / gamma], dtype=torch.float32)
        _, gi = ref_wa.forward(pin, c(d.flat_net2pin_map), c(d.flat_net2pin_start_map), c(d.pin2net_map),
                               c(d.net_weights), c(mask), ig)
        gw = ref_wa.backward(torch.ones(1), pin, gi, c(d.flat_net2pin_map), c(d.flat_net2pin_start_map),
                             c(d.pin2net_map), c(d.net_weights), c(mask), ig)
        pm = c(d.pin2node_map >= d.num_movable_nodes)
        gw[:d.num_pins].masked_fill_(pm, 0.0)
        gw[d.num_pins:].masked_fill_(pm, 0.0)
        gref = ref_pp.backward(gw, c(pos_np), c(d.pin_offset_x), c(d.pin_offset_y), p2n, c(d.flat_node2pin_map),
                               c(d.flat_node2pin_start_map), d.num_physical_nodes).numpy()
        assert np.max(np.abs(grad - gref)) <= 1e-5 * np.max(np.abs(gref))


def test_density_adjoint_against_fd_and_reference(setup):
    from dreamplace_b200.electric_potential import ElectricPotential
    from dreamplace_b200.dct2_fft2 import cos_matrix, icos_matrix, isin_matrix
    d, pos_np, cells = setup
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    m = d.num_movable_nodes
    sorted_map = t(np.argsort(d.node_size_x[:m], kind="stable").astype(np.int32))
    op = ElectricPotential(t(d.node_size_x), t(d.node_size_y), t(d.bin_centers(d.xl, d.xh, d.bin_size_x)),
                           t(d.bin_centers(d.yl, d.yh, d.bin_size_y)), d.target_density, d.xl, d.yl, d.xh, d.yh,
                           d.bin_size_x, d.bin_size_y, m, d.num_terminals, d.num_filler_nodes, 0, True, sorted_map,
                           precision="fp32")
    pos = t(pos_np).requires_grad_(True)
    op(pos).backward()
    grad = pos.grad.double().cpu().numpy()
    # (the kernel equals the reference CPU electric_force bit for bit on the same
    # field maps: tests/test_gpu_ops.py::test_electric_force_bit_exact)
    # fp64 finite differences of the energy
    M, N = d.num_bins_x, d.num_bins_y
    s = oracle.stretched(d.node_size_x, d.node_size_y, d.bin_size_x, d.bin_size_y)
    init = op.initial_density_map.double()
    wu = torch.arange(M, dtype=F64, device=dev).mul(2 * np.pi / M).view(M, 1)
    wv = torch.arange(N, dtype=F64, device=dev).mul(2 * np.pi / N).view(1, N) * (d.bin_size_x / d.bin_size_y)
    w2 = wu ** 2 + wv ** 2
    w2[0, 0] = 1.0
    inv = 1.0 / w2
    inv[0, 0] = 0.0
    mats = [t(f(k)) for f, k in ((cos_matrix, M), (icos_matrix, M), (isin_matrix, M), (cos_matrix, N),
                                 (icos_matrix, N), (isin_matrix, N))] + [inv]
    n = d.num_nodes
    p64 = t(pos_np.astype(np.float64))
    base = density_fp64(d, p64, s)
    hstep = 1e-3 * d.bin_size_x
    fd, got = [], []
    for c in cells[:64]:
        for axis in (0, 1):
            i = axis * n + int(c)
            pp_, pm_ = p64.clone(), p64.clone()
            pp_[i] += hstep
            pm_[i] -= hstep
            ep_ = energy_fp64(d, density_fp64(d, pp_, s), init, mats)
            em_ = energy_fp64(d, density_fp64(d, pm_, s), init, mats)
            bs = d.bin_size_x if axis == 0 else d.bin_size_y
            expected = 2.0 / (d.bin_size_x * d.bin_size_y * bs)
            fd.append(float(ep_ - em_) / (2 * hstep) / expected)
            got.append(grad[i])
    fd, got = np.array(fd), np.array(got)
    cos = float(np.dot(fd, got) / (np.linalg.norm(fd) * np.linalg.norm(got)))
    scale = float(np.dot(fd, got) / np.dot(got, got))
    print("density FD vs field force: cosine %.4f, scale %.4f (expected 1)" % (cos, scale))
    assert cos > 0.9, cos
    assert abs(scale - 1.0) < 0.25, scale
    del base


@pytest.mark.parametrize("precision", ["fp32", "split_bf16"])
def test_recomputed_field_matches_stored(setup, precision):
    """recompute_field=True (forward keeps only rho, backward repeats the
    solve) gives the stored-field gradient bit for bit and the same energy."""
    from dreamplace_b200.electric_potential import ElectricPotential
    d, pos_np, _ = setup
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    m = d.num_movable_nodes
    sorted_map = t(np.argsort(d.node_size_x[:m], kind="stable").astype(np.int32))
    out = []
    for recompute in (False, True):
        op = ElectricPotential(t(d.node_size_x), t(d.node_size_y), t(d.bin_centers(d.xl, d.xh, d.bin_size_x)),
                               t(d.bin_centers(d.yl, d.yh, d.bin_size_y)), d.target_density, d.xl, d.yl, d.xh,
                               d.yh, d.bin_size_x, d.bin_size_y, m, d.num_terminals, d.num_filler_nodes, 0, True,
                               sorted_map, fast_mode=False, precision=precision, recompute_field=recompute)
        pos = t(pos_np).requires_grad_(True)
        energy = op(pos)
        energy.backward()
        out.append((float(energy.detach()), pos.grad.clone()))
    (e0, g0), (e1, g1) = out
    assert torch.equal(g0, g1)
    assert abs(e0 - e1) <= 1e-6 * abs(e0), (e0, e1)
