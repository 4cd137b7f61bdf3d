"""dp_density_map_fx64_noalloc through the C ABI: the allocation-free
deterministic scatter for callers that cannot allocate device memory
(fixed-budget hosts, FFI hosts without the CUDA allocator).  Its output must
equal dp_density_map_fx64's (which takes a caller-owned scratch map) bit for
bit -- the fixed-point map is exact -- on two calls in a row, since every call
reuses the same built-in scratch array.  The file is named to be collected
last; the test passes both in a fresh process
(``pytest tests/test_zz_no_alloc.py``) and after the other tests."""
import ctypes
import math
import os

import numpy as np
import pytest
import torch

from dreamplace_b200 import synthetic

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "dreamplace_b200", "lib", "libdreamplace_b200.so")


def test_noalloc_scatter_matches_scratch_entry_point():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = ctypes.CDLL(LIB)
    lib.dp_last_error.restype = ctypes.c_char_p
    d = synthetic.cells_10k()
    pos_np = d.initial_positions()
    rng = np.random.RandomState(4)
    n, m = d.num_nodes, d.num_movable_nodes
    pos_np[:m] = rng.uniform(d.xl, d.xh - 32, size=m)
    pos_np[n:n + m] = rng.uniform(d.yl, d.yh - 12, size=m)
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    pos = t(pos_np)
    sx, sy = t(d.node_size_x), t(d.node_size_y)
    sxc = sx.clamp(min=d.bin_size_x * math.sqrt(2))
    syc = sy.clamp(min=d.bin_size_y * math.sqrt(2))
    ox, oy = (sx - sxc).mul(0.5), (sy - syc).mul(0.5)
    ratio = sx * sy / (sxc * syc)
    init = torch.rand(d.num_bins_x * d.num_bins_y, device=dev)
    nbins = d.num_bins_x * d.num_bins_y
    die = (d.xh - d.xl) * (d.yh - d.yl)
    fb = max(64 - max(int(math.ceil(math.log2(die))) + 1, 32), 0)
    P, F, I = ctypes.c_void_p, ctypes.c_float, ctypes.c_int
    common = [P(pos.data_ptr()), I(n), P(sxc.data_ptr()), P(syc.data_ptr()), P(ox.data_ptr()), P(oy.data_ptr()),
              P(ratio.data_ptr()), P(init.data_ptr()), F(d.xl), F(d.yl), F(d.xh), F(d.yh), F(d.bin_size_x),
              F(d.bin_size_y), F(1.0 / d.bin_size_x), F(1.0 / d.bin_size_y), I(m), I(d.num_filler_nodes),
              I(d.num_bins_x), I(d.num_bins_y), P(None), I(fb)]
    stream = P(torch.cuda.current_stream().cuda_stream)
    scratch = torch.empty(nbins, dtype=torch.int64, device=dev)
    ref = torch.empty(nbins, device=dev)
    rc = lib.dp_density_map_fx64(*common, P(scratch.data_ptr()), P(ref.data_ptr()), stream)
    assert rc == 0, lib.dp_last_error()
    for _ in range(2):
        out = torch.full((nbins,), float("nan"), device=dev)
        rc = lib.dp_density_map_fx64_noalloc(*common, P(out.data_ptr()), stream)
        assert rc == 0, lib.dp_last_error()
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
    # grids beyond the built-in scratch are rejected before any launch
    big = list(common)
    big[18], big[19] = I(2048), I(1024)
    rc = lib.dp_density_map_fx64_noalloc(*big, P(out.data_ptr()), stream)
    assert rc == -1 and b"exceed" in lib.dp_last_error()
