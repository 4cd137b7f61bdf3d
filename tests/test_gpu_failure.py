"""Failure detection without a GPU fault.

* The tensor-core GEMM's bounded waits: with the host-set test hook the TMA
  producer issues no copy, so the MMA warp's wait on the first stage runs out
  after a short host-set budget; the launch returns, dp_tc_status reports the
  expired wait, and the context stays usable (the next solve's field maps equal
  the ones before the failure bit for bit).
* GP divergence rollback (reference dreamplace/NonLinearPlace.py:534-570,
  641-651): late in GP the movable cells' positions are permuted on the host
  (the occupied spots stay, every net is torn apart), the HPWL jumps while the
  overflow holds, the divergence check fires within its 50-iteration window,
  the loop rolls back to the best position recorded, evaluates it and stops.
"""
import math

import numpy as np
import pytest
import torch

from dreamplace_b200 import synthetic
from dreamplace_b200.nonlinear_place import NonLinearPlace
from dreamplace_b200.params import Params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def C():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dreamplace_b200._native import C
    return C


def _solve(M, precision):
    from dreamplace_b200.electric_potential import poisson_solve
    rng = np.random.RandomState(3)
    rho = torch.from_numpy(rng.uniform(0, 1, size=(M, M)).astype(np.float32)).cuda()
    ex, ey, energy = poisson_solve(rho, 10.0, 10.0, precision)
    torch.cuda.synchronize()
    return ex.clone(), ey.clone(), energy.clone()


def test_gemm_bounded_wait_expires_and_context_survives(C):
    before = _solve(128, "split_bf16")
    assert C.tc_status() == 0
    try:
        C.tc_set_wait_budget(20_000_000)  # ~10 ms
        C.tc_set_skip_loads(1)
        _solve(128, "split_bf16")
        status = C.tc_status()
    finally:
        C.tc_set_skip_loads(0)
        C.tc_set_wait_budget(4_000_000_000)
    assert status == 2  # the MMA warp's wait for the first operand stage ran out
    # the context stays usable: the next solve equals the one before (field
    # maps bit for bit; the energy's per-CTA fp64 partials are added atomically)
    after = _solve(128, "split_bf16")
    assert C.tc_status() == 0
    assert torch.equal(before[0], after[0]) and torch.equal(before[1], after[1])
    assert math.isclose(float(before[2]), float(after[2]), rel_tol=1e-12)


@pytest.mark.parametrize("engine", ["graph", "autograd"])
def test_divergence_rollback_after_host_injection(C, engine):
    d = synthetic.cells_10k()
    p = Params(target_density=d.target_density, stop_overflow=0.07, dct_precision="fp32", gp_engine=engine,
               deterministic_flag=1)
    placer = NonLinearPlace(p, d)
    rng = np.random.RandomState(5)
    state = {"injected": None, "best_hpwl": None}
    m, n = d.num_movable_nodes, d.num_nodes

    def cb(it, metric):
        if state["injected"] is None and metric.overflow < 0.2:
            pos = placer.stepper.position().detach().clone()
            perm = torch.from_numpy(rng.permutation(m)).cuda()
            pos[:m] = pos[:m][perm]
            pos[n:n + m] = pos[n:n + m][perm]
            placer.stepper.set_position(pos)
            state["injected"] = it

    metrics = placer(p, d, callback=cb)
    flat = [x for g in metrics for lam in g for x in lam]
    assert state["injected"] is not None
    assert placer.divergence_iteration is not None
    assert state["injected"] < placer.divergence_iteration <= state["injected"] + 60
    # the injection tore the nets apart: the HPWL jumped
    k = state["injected"]
    assert max(x.hpwl for x in flat[k + 1:]) > 1.5 * flat[k].hpwl
    # the rollback iteration evaluates the best position recorded (the lowest
    # overflow so far) and the loop stops after it, as the reference's does
    assert flat[-1].iteration == placer.divergence_iteration
    best = placer.best["metric"]
    assert math.isclose(flat[-1].hpwl, best.hpwl, rel_tol=1e-9), (flat[-1].hpwl, best.hpwl)
    assert math.isclose(flat[-1].overflow, best.overflow, rel_tol=1e-9)
