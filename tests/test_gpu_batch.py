"""Batched placement (several designs interleaved on one GPU, one stream each):
every design follows exactly the trajectory it follows alone (deterministic
density maps), and all of them reach the overflow stop."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_batched_designs_match_single_runs():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dreamplace_b200 import batch
    designs = batch.batch_set(3, seed=3, lo=3000, hi=8000)
    res_b, _ = batch.BatchPlacer(designs, deterministic=1).run(max_iterations=40)
    res_s, _ = batch.BatchPlacer(designs, deterministic=1).run_sequential(max_iterations=40)
    for rb, rs in zip(res_b, res_s):
        tb = [(m.hpwl, m.overflow) for g in rb for lam in g for m in lam]
        ts = [(m.hpwl, m.overflow) for g in rs for lam in g for m in lam]
        assert tb == ts
    full, _ = batch.BatchPlacer(designs).run()
    assert all(r[-1][-1][-1].overflow <= 0.07 + 1e-9 for r in full)
