"""Checkpoint / resume of global placement (the graph engine's GP loop): a
run saves its state every 40 iterations; a new placer resumed from the state
at iteration 40 (through a torch.save / torch.load round trip) follows the
original run's trajectory bit for bit in deterministic mode and ends at the
same positions.  (The reference dumps the placement and keeps an optimizer
state copy for restarts: dreamplace/BasicPlace.py:1174-1248,
dreamplace/NonLinearPlace.py:273.)"""
import io

import pytest
import torch

from dreamplace_b200 import synthetic
from dreamplace_b200.nonlinear_place import NonLinearPlace
from dreamplace_b200.params import Params

pytestmark = pytest.mark.gpu


def test_resume_follows_the_original_trajectory():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    d = synthetic.cells_10k()
    p = Params(target_density=d.target_density, stop_overflow=0.07, dct_precision="split_bf16", deterministic_flag=1)
    saved = {}
    rows_a, rows_b = [], []
    a = NonLinearPlace(p, d)
    a(p, d, max_iterations=90, callback=lambda it, m: rows_a.append((it, m.hpwl, m.overflow, m.max_density)),
      checkpoint_every=40, checkpoint_fn=lambda st: saved.__setitem__(st["loop"]["iteration"], st))
    assert sorted(saved) == [40, 80]
    buf = io.BytesIO()
    torch.save(saved[40], buf)
    buf.seek(0)
    state = torch.load(buf, weights_only=False)
    b = NonLinearPlace(p, d)
    b(p, d, max_iterations=90, callback=lambda it, m: rows_b.append((it, m.hpwl, m.overflow, m.max_density)),
      resume=state)
    assert len(rows_a) == 90 and rows_b == rows_a[40:]
    assert torch.equal(a.pos[0].data, b.pos[0].data)
    with pytest.raises(ValueError):
        c = NonLinearPlace(Params(target_density=d.target_density, gp_engine="autograd"), d)
        c(c.params, d, max_iterations=2, resume=state)
