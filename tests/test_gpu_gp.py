"""Full global placement on the GPU (CPU-runnable design, 10k cells, 128x128 bins).

* the graph-captured engine and the reference-shaped autograd path follow the
  same trajectory (same kernels, same operation order) for the first iterations;
* GP reaches the 0.07 overflow stop, and the split-BF16 Poisson solve ends
  within 0.1% HPWL of the plain fp32 form."""
import pytest
import torch

from dreamplace_b200 import synthetic
from dreamplace_b200.nonlinear_place import place
from dreamplace_b200.params import Params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def design():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return synthetic.cells_10k()


def run(design, engine, precision, iters=None, deterministic=0):
    traj = []
    p = Params(target_density=design.target_density, stop_overflow=0.07, dct_precision=precision, gp_engine=engine,
               deterministic_flag=deterministic)
    placer, res = place(design, p, max_iterations=iters, callback=lambda it, m: traj.append((m.hpwl, m.overflow)))
    return placer, res, traj


def test_engine_matches_autograd_path(design):
    _, _, a = run(design, "autograd", "fp32", 8, deterministic=1)
    _, _, b = run(design, "graph", "fp32", 8, deterministic=1)
    _, _, c = run(design, "eager", "fp32", 8, deterministic=1)
    for (ha, oa), (hb, ob), (hc, oc) in zip(a, b, c):
        assert abs(ha - hb) <= 1e-4 * ha and abs(oa - ob) <= 1e-4
        assert hb == hc and ob == oc  # graph replay == the same kernels launched eagerly


def test_gp_converges_and_split_bf16_matches_plain(design):
    """Deterministic mode (int64 density maps), so the two runs differ only in
    the Poisson-solve arithmetic."""
    _, plain, _ = run(design, "graph", "fp32", deterministic=1)
    _, split, _ = run(design, "graph", "split_bf16", deterministic=1)
    for r in (plain, split):
        assert r["overflow"] <= 0.07 + 1e-9 and r["iterations"] < 1000
    print("plain", plain, "split", split, "rel", abs(split["hpwl"] - plain["hpwl"]) / plain["hpwl"])
    assert abs(split["hpwl"] - plain["hpwl"]) <= 1e-3 * plain["hpwl"], (split, plain)


def test_recapture_with_one_timed_piece_keeps_the_trajectory(design):
    """GPEngine.time_only (the bench's timed window): the trial graphs,
    captured again mid-GP with one piece's events, follow the run that kept
    its first graphs bit for bit (deterministic mode), and the piece is timed."""
    p = lambda **kw: Params(target_density=design.target_density, stop_overflow=0.07,  # noqa: E731
                            dct_precision="split_bf16", deterministic_flag=1, **kw)
    t1, t2 = [], []
    place(design, p(time_pieces=True), max_iterations=40, callback=lambda it, m: t1.append((m.hpwl, m.overflow)))
    holder = {}

    def cb(it, m):
        t2.append((m.hpwl, m.overflow))
        if it == 12:
            eng = holder["placer"].stepper.eng
            eng.time_only(["wa_forward"])
            holder["eng"] = eng

    from dreamplace_b200.nonlinear_place import NonLinearPlace
    params = p(time_pieces=True)
    placer = NonLinearPlace(params, design, "cuda")
    holder["placer"] = placer
    placer(params, design, max_iterations=40, callback=cb)
    assert t1 == t2
    means = holder["eng"].piece_means()
    assert set(means) == {"wa_forward"} and means["wa_forward"] > 0


def test_gp_deterministic_mode_is_reproducible(design):
    p = lambda: Params(target_density=design.target_density, stop_overflow=0.07, dct_precision="fp32",  # noqa: E731
                       deterministic_flag=1)
    t1, t2 = [], []
    place(design, p(), max_iterations=30, callback=lambda it, m: t1.append((m.hpwl, m.overflow)))
    place(design, p(), max_iterations=30, callback=lambda it, m: t2.append((m.hpwl, m.overflow)))
    assert t1 == t2


def test_trial_metrics_match_direct_evaluation(design):
    """The HPWL summed inside the trial's WA forward and the overflow from the
    trial's movable-only map equal a direct evaluation of the same position
    (bit for bit in deterministic mode), and the HPWL matches the oracle."""
    import numpy as np
    import oracle
    placer, _, _ = run(design, "graph", "fp32", 6, deterministic=1)
    eng = placer.stepper.eng
    q = eng.parity  # v_k, produced by the last accepted trial
    h_trial, o_trial = eng.H[q][0].item(), eng.O[q][0:2].clone()
    eng.evaluate(q)
    assert eng.H[q][0].item() == h_trial
    assert torch.equal(eng.O[q][0:2], o_trial)
    d = design
    pos = eng.V[q].cpu().numpy()
    n, P = d.num_nodes, d.num_pins
    px = pos[d.pin2node_map] + d.pin_offset_x
    py = pos[n + d.pin2node_map] + d.pin_offset_y
    ref = oracle.hpwl(np.concatenate([px, py]).astype(np.float32), d.flat_net2pin_map, d.flat_net2pin_start_map,
                      np.ones(d.num_nets, np.uint8), d.net_weights)
    ref = ref[0] if isinstance(ref, tuple) else ref
    assert abs(h_trial - ref) <= 1e-6 * ref


def test_iteration_head_matches_host_loop():
    """dp_iteration_head against the host loop's formulas (NonLinearPlace
    density-weight update in RePlAce HPWL mode, gamma update, Nesterov advance):
    HPWL up and down, both clamps of mu, the first iteration (no update)."""
    import math
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dreamplace_b200._native import C
    base_gamma, area, ref, lower, upper = 4.0 * 46.875, 2.5e6, 350000.0, 0.95, 1.05
    cases = [(0, 1.0e6, 9.0e5, 0.9), (1, 1.0e6, 9.0e5, 0.5), (7, 1.0e6, 1.1e6, 0.3), (12, 1.0e6, 1.0e6 + 1e9, 0.12),
             (30, 2.0e6, 2.0e6 + 1.0, 0.07), (400, 5.0e5, 4.0e5, 0.2)]
    for k, hp_prev, hp, ovf in cases:
        st_prev = torch.zeros(8 + 2 * 1280, dtype=torch.float64, device="cuda")
        st_prev[0:4] = torch.tensor([0.3, 2.5, 3.1, 0.4], dtype=torch.float64)
        st_new = torch.zeros_like(st_prev)
        sched_prev = torch.tensor([float(k), hp_prev], dtype=torch.float64, device="cuda")
        sched_new = torch.zeros(2, dtype=torch.float64, device="cuda")
        w_prev = torch.tensor([1.7e-4, 20.0, 0.05], dtype=torch.float32, device="cuda")
        w_new = torch.zeros(3, dtype=torch.float32, device="cuda")
        hpk = torch.tensor([hp], dtype=torch.float64, device="cuda")
        ovk = torch.tensor([ovf * area], dtype=torch.float64, device="cuda")
        C.iteration_head(st_prev, st_new, sched_prev, sched_new, hpk, ovk, w_prev, w_new, base_gamma, area, ref,
                         lower, upper)
        # the host loop (nonlinear_place.py run_gen)
        f = k + 1
        lam = torch.tensor([1.7e-4], dtype=torch.float32)
        if f > 1:
            delta = hp - hp_prev
            if delta < 0:
                mu = upper * max(math.pow(0.9999, float(f)), 0.98)
            else:
                mu = upper * min(max(math.pow(upper, -delta / ref), lower), upper)
            lam.mul_(mu)
        gamma = torch.zeros((), dtype=torch.float32).fill_(base_gamma * math.pow(10, ((ovf * area) / area - 0.1) * 20 / 9 - 1))
        w = w_new.cpu()
        assert w[0].item() == lam.item(), (k, w[0].item(), lam.item())
        assert w[1].item() == gamma.item()
        assert w[2].item() == (1.0 / gamma.reshape(1)).item()
        a = 3.1
        an = (1.0 + math.sqrt(4.0 * a * a + 1.0)) / 2.0
        got = st_new[0:4].cpu().tolist()
        assert got == [0.3, a, an, (a - 1.0) / an]
        assert sched_new.cpu().tolist() == [float(f), hp]


def test_speculative_iterations_match_serial(design):
    """Iteration k+1 enqueued ahead of the host (speculate) gives the serial
    loop's trajectory bit for bit in deterministic mode, retries included."""
    traj = {}
    for spec in (False, True):
        t = []
        p = Params(target_density=design.target_density, stop_overflow=0.07, dct_precision="fp32",
                   deterministic_flag=1, speculate=spec)
        placer, res = place(design, p, max_iterations=120, callback=lambda it, m: t.append((m.hpwl, m.overflow)))
        traj[spec] = (t, placer.stepper.eng.trials, placer.pos[0].detach().cpu())
    (t0, n0, p0), (t1, n1, p1) = traj[False], traj[True]
    assert n0 == n1 and n0 > 120  # some iterations needed a retry
    assert t0 == t1
    assert torch.equal(p0, p1)


def test_trial_gate_skips_gated_kernels():
    """Launches made while a trial gate is installed return at once when the
    word is set, and run when it is clear; dp_trial_gate sets it from an
    accept flag; launches after removal ignore the word."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dreamplace_b200._native import C
    n = 1000
    xy = torch.arange(2 * n, dtype=torch.float32, device="cuda")
    order = torch.arange(n - 1, -1, -1, dtype=torch.int32, device="cuda")
    gate = torch.zeros(1, dtype=torch.int32, device="cuda")
    rejected = torch.zeros(1, dtype=torch.float64, device="cuda")
    accepted = torch.ones(1, dtype=torch.float64, device="cuda")
    out = torch.full((2 * n,), -1.0, device="cuda")
    C.set_trial_gate(gate)
    try:
        C.trial_gate(gate, rejected)
        C.gather_order_xy(xy, order, n, out)
        assert gate.item() == 1 and bool((out == -1.0).all())
        C.trial_gate(gate, accepted)
        C.gather_order_xy(xy, order, n, out)
        assert gate.item() == 0
        assert torch.equal(out.view(-1, 2), xy.view(-1, 2)[order.long()])
        C.trial_gate(gate, rejected)
    finally:
        C.set_trial_gate(None)
    out.fill_(-1.0)
    C.gather_order_xy(xy, order, n, out)  # gate removed: runs although the word is set
    assert gate.item() == 1 and torch.equal(out.view(-1, 2), xy.view(-1, 2)[order.long()])


@pytest.mark.parametrize("xyo_mode,wa_grad_order", [("order", "lane"), ("trial", "lane"), ("gather", "csr")])
def test_engine_layout_options_give_the_same_trajectory(design, xyo_mode, wa_grad_order):
    """The engine's layout options (how the scatter reads the trial point, where
    the WA gradient is written) change no arithmetic: deterministic runs give
    the default layout's trajectory bit for bit."""
    def traj(**kw):
        t = []
        p = Params(target_density=design.target_density, stop_overflow=0.07, dct_precision="fp32",
                   deterministic_flag=1, **kw)
        place(design, p, max_iterations=40, callback=lambda it, m: t.append((m.hpwl, m.overflow, m.objective)))
        return t
    assert traj(xyo_mode=xyo_mode, wa_grad_order=wa_grad_order) == traj()


def test_best_position_copied_before_its_slot_is_reused(design):
    """The GP loop's best position is copied lazily: a newer best supersedes a
    pending copy, a pending copy is made on the stream before a trial
    overwrites the slot holding it, and the divergence rollback
    (set_position) completes it first."""
    p = Params(target_density=design.target_density, stop_overflow=0.07, dct_precision="fp32", deterministic_flag=1)
    placer, _ = place(design, p, max_iterations=10)
    eng = placer.stepper.eng

    def step():
        g = eng.step_gen()
        next(g)
        try:
            next(g)
        except StopIteration:
            pass

    step()
    first = eng.current_position().clone()
    buf = eng.mark_best(None)
    step()
    second = eng.current_position().clone()
    assert eng.mark_best(buf) is buf  # supersedes the first best before any copy
    for _ in range(4):
        step()  # the trials write every slot, the second best's included
    torch.cuda.synchronize()
    assert eng.best_slot is None
    assert torch.equal(buf, second) and not torch.equal(buf, first)
    step()
    third = eng.current_position().clone()
    eng.mark_best(buf)
    eng.set_position(buf)  # completes the pending copy, then restores from it
    torch.cuda.synchronize()
    assert torch.equal(buf, third) and torch.equal(eng.current_position(), third)


def test_profile_piece_runs_every_piece():
    """The profiling entry point runs each piece of the trial on a GP state."""
    from dreamplace_b200 import profile_piece
    for piece in profile_piece.PIECES:
        profile_piece.main(["--piece", piece, "--design", "cells_10k", "--iterations", "3", "--repeat", "1"])
