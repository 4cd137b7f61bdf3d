"""Global placement driver.

Mirrors the reference's ``NonLinearPlace.__call__`` for the default flow
(dreamplace/NonLinearPlace.py:49-798): one stage, nesterov, the three nested
loops Lgamma / Llambda / Lsub with their stop criteria, per-iteration HPWL and
overflow evaluation (dreamplace/EvalMetrics.py:100-141), density-weight and
gamma updates, best-position tracking, divergence rollback and the plateau
rule that turns on the quadratic density penalty and, when overflow stays
above 0.95, injects entropy (shrink towards the centroid plus noise).

Two executions of the same iteration:

* ``params.gp_engine = "graph"`` (default): ``engine.GPEngine`` -- fused
  kernels, no autograd, one CUDA-graph replay per Nesterov trial;
* ``params.gp_engine = "autograd"``: the reference-shaped path through the
  drop-in ops, ``torch.autograd`` and ``nesterov.NesterovAcceleratedGradientOptimizer``.

The per-iteration metrics (HPWL and overflow in fp64) are read back once per
iteration in both.
"""
import logging
import math
import time

import numpy as np
import torch
from torch import nn

from .engine import GPEngine
from .nesterov import NesterovAcceleratedGradientOptimizer
from .params import Params
from .place_obj import PlaceDataCollection, PlaceObj, build_ops

logger = logging.getLogger(__name__)


class EvalMetrics(object):
    """Per-iteration metrics (reference dreamplace/EvalMetrics.py); host floats."""

    def __init__(self, iteration, hpwl, overflow, max_density, objective=None):
        self.iteration = iteration
        self.hpwl = hpwl
        self.overflow = overflow
        self.max_density = max_density
        self.objective = objective
        self.gamma = None
        self.density_weight = None

    @property
    def _host(self):
        return (self.hpwl, self.overflow, self.max_density)

    def __str__(self):
        return "iteration %4d, HPWL %.6E, Overflow %.6E, MaxDensity %.3E" % (self.iteration, self.hpwl,
                                                                            self.overflow, self.max_density)


class _AutogradStepper(object):
    """The reference-shaped iteration: drop-in ops + autograd + Nesterov optimizer."""

    def __init__(self, placer, model, params, design, lr0):
        self.placer, self.model, self.params, self.design = placer, model, params, design
        self.pos = placer.data_collections.pos[0]
        self.opt = NesterovAcceleratedGradientOptimizer(placer.parameters(), lr=0.0,
                                                        obj_and_grad_fn=model.obj_and_grad_fn,
                                                        constraint_fn=placer.op_collections.move_boundary_op)
        if params.gp_noise_ratio > 0.0:
            model.ops.noise_op(self.pos, params.gp_noise_ratio)
        lr = model.estimate_initial_learning_rate(self.pos, lr0)
        for g in self.opt.param_groups:
            g["lr"] = lr.data

    def step(self, first):
        m, ops, d = self.model, self.placer.op_collections, self.design
        pos = self.pos
        ops.move_boundary_op(pos)
        if float(m.density_weight.mean()) == 0.0:
            m.initialize_density_weight(self.params, d)
        self.opt.zero_grad(set_to_none=False)
        with torch.no_grad():
            hp = ops.hpwl_f64_op(pos)[0]
            ovf = ops.density_overflow_op.overflow_f64(pos)
        self.opt.step()
        obj = self.opt.param_groups[0]["obj_k_1"][0]
        v = torch.stack([hp.reshape(()), ovf[0], ovf[1], obj.reshape(()).double()]).cpu().numpy()
        return float(v[0]), float(v[1]) / d.total_movable_node_area, float(v[2]), float(v[3])

    def position(self):
        return self.pos.data

    def set_position(self, t):
        self.pos.data.copy_(t)


class _EngineStepper(object):
    """The graph-captured iteration of engine.GPEngine."""

    def __init__(self, placer, model, params, design, lr0, use_graphs, resume=None):
        self.model, self.params, self.design = model, params, design
        pos = placer.data_collections.pos[0]
        ep = model.ops.density_op
        if ep.initial_density_map is None:
            ep.compute_initial_density_map(pos.data)
        ov = model.ops.density_overflow_op
        if ov.initial_density_map is None:
            ov.compute_initial_density_map(pos.data)
        self.eng = GPEngine(params, design, placer.data_collections, placer.op_collections, model, use_graphs)
        if resume is not None:
            # the optimizer is already set up: its state comes from the checkpoint
            self.lr = resume["lr"]
            self.eng.load_state_dict(resume["engine"])
            return
        if params.gp_noise_ratio > 0.0:
            model.ops.noise_op(self.eng.V[0], params.gp_noise_ratio)
        self.lr = self.eng.initial_learning_rate(lr0)

    def step(self, first):
        gen = self.step_gen(first)
        try:
            while True:
                next(gen)
        except StopIteration as stop:
            return stop.value

    def step_gen(self, first):
        """step() as a generator that yields once the iteration's first trial is
        enqueued (see GPEngine.step_gen)."""
        e = self.eng
        if first:
            e.move_boundary(e.V[e.parity])
            e.initialize_density_weight()
            e.start_optimizer(self.lr)
        h, o, md, obj, trials = yield from e.step_gen()
        return h, o, md, obj

    device_updates = True

    def sync_model(self):
        self.eng.sync_model()

    def position(self):
        return self.eng.current_position()

    def set_position(self, t):
        self.eng.set_position(t)

    def record_best(self, buf):
        return self.eng.mark_best(buf)

    def best_position(self):
        return self.eng.flush_best()


class NonLinearPlace(nn.Module):
    """Global placement of one design on one GPU."""

    def __init__(self, params, design, device=None):
        super().__init__()
        self.params = params
        self.design = design
        self.device = torch.device(device or "cuda")
        np.random.seed(params.random_seed)
        init = design.initial_positions(seed=params.random_seed)
        self.pos = nn.ParameterList([nn.Parameter(torch.from_numpy(init).to(self.device))])
        self.data_collections = PlaceDataCollection(self.pos, params, design, self.device)
        self.op_collections = build_ops(params, design, self.data_collections)

    def __call__(self, params=None, design=None, max_iterations=None, callback=None, checkpoint_every=0,
                 checkpoint_fn=None, resume=None):
        gen = self.run_gen(params, design, max_iterations, callback, checkpoint_every, checkpoint_fn, resume)
        try:
            while True:
                next(gen)
        except StopIteration as stop:
            return stop.value

    def run_gen(self, params=None, design=None, max_iterations=None, callback=None, checkpoint_every=0,
                checkpoint_fn=None, resume=None):
        """The GP loop as a generator: with the graph engine it yields once per
        iteration, after enqueuing the iteration's first trial, so that a batch
        driver can interleave several designs (each on its own stream); the
        return value is __call__'s.

        Checkpoint / resume (graph engine, the default schedule): with
        checkpoint_every = N, checkpoint_fn(state) receives, at the start of
        every N-th iteration, the loop's and the engine's state (host tensors
        and plain values, torch.save-able); resume=state continues a run from
        such a state with the same trajectory.  The state plays the role of the
        reference's dumped placement plus optimizer state
        (dreamplace/BasicPlace.py:1174-1248, NonLinearPlace.py:273)."""
        params = params or self.params
        design = design or self.design
        torch.manual_seed(params.random_seed)
        # the entropy injection's noise comes from a generator of this run, so
        # designs placed together (interleaved on one GPU) draw the noise they
        # draw alone
        noise_gen = torch.Generator(device=self.device)
        noise_gen.manual_seed(params.random_seed + 1)
        gp = dict(params.global_place_stages[0])
        if max_iterations is not None:
            gp["iteration"] = max_iterations
        model = PlaceObj(0.0, params, design, self.data_collections, self.op_collections, gp).to(self.device)
        self.model = model
        mode = getattr(params, "gp_engine", "graph")
        if (checkpoint_every or resume is not None) and mode != "graph":
            raise ValueError("checkpoint / resume runs on the graph engine (gp_engine='graph')")
        if resume is not None:
            self._restore_model(model, resume)
        if mode == "autograd":
            stepper = _AutogradStepper(self, model, params, design, gp["learning_rate"])
        else:
            stepper = _EngineStepper(self, model, params, design, gp["learning_rate"], mode == "graph", resume)
        self.stepper = stepper
        # the graph engine applies the density-weight and gamma updates itself,
        # on the device at the start of the next iteration (the same formulas)
        device_updates = getattr(stepper, "device_updates", False)
        base_gamma = model.base_gamma(params, design)
        ref_hpwl = params.RePlAce_ref_hpwl
        lower, upper = params.RePlAce_LOWER_PCOF, params.RePlAce_UPPER_PCOF
        all_metrics = []
        best = {"metric": None, "pos": None}
        overflow_list = [1.0]
        divergence_list = []
        last_perturb_iter = -50
        stop_placement = False
        iteration = 0
        flat_llambda = 0
        start_step = 0
        self.iteration_times = []
        self.divergence_iteration = None  # the iteration whose divergence check rolled back, if any
        if resume is not None:
            L = resume["loop"]
            iteration = start_step = int(L["iteration"])
            flat_llambda = int(L["flat_llambda"])
            last_perturb_iter = int(L["last_perturb_iter"])
            overflow_list = list(L["overflow_list"])
            divergence_list = [list(x) for x in L["divergence_list"]]
            all_metrics = [[[EvalMetrics(*row)]] for row in L["metrics"]]
            bm = L["best_metric"]
            best = {"metric": EvalMetrics(*bm) if bm is not None else None,
                    "pos": L["best_pos"].to(self.device) if L["best_pos"] is not None else None}
            noise_gen.set_state(L["noise_gen"])
            self.iteration_times = list(L.get("iteration_times", []))

        def checkpoint():
            flat = [m for g in all_metrics for lam in g for m in lam]
            eng_state = stepper.eng.state_dict()
            best_pos = stepper.best_position() if best["metric"] is not None else None
            return {"loop": {"iteration": iteration, "flat_llambda": flat_llambda,
                             "last_perturb_iter": last_perturb_iter, "overflow_list": list(overflow_list),
                             "divergence_list": [list(x) for x in divergence_list],
                             "metrics": [(m.iteration, m.hpwl, m.overflow, m.max_density, m.objective)
                                         for m in flat],
                             "best_metric": None if best["metric"] is None else
                             (best["metric"].iteration, best["metric"].hpwl, best["metric"].overflow,
                              best["metric"].max_density, best["metric"].objective),
                             "best_pos": None if best_pos is None else best_pos.detach().cpu().clone(),
                             "noise_gen": noise_gen.get_state(), "iteration_times": list(self.iteration_times)},
                    "model": {"density_factor": model.density_factor, "quad_penalty": model.quad_penalty,
                              "init_density": None if model.init_density is None else model.init_density.cpu(),
                              "density_weight": model.density_weight.detach().cpu(),
                              "gamma": model.gamma.detach().cpu()},
                    "engine": eng_state, "lr": stepper.lr}

        def divergence_numpy(xs, threshold):
            x = np.array(xs)
            overflow_mean = np.mean(x[:, 1])
            overflow_diff = np.sum(np.maximum(0, np.sign(x[1:, 1] - x[:-1, 1]))) / (x.shape[0] - 1)
            overflow_range = np.max(x[:, 1]) - np.min(x[:, 1])
            wl_mean = np.mean(x[:, 0])
            bh, bo = best["metric"].hpwl, best["metric"].overflow
            wl_ratio = (wl_mean - bh) / bh
            overflow_ratio = (overflow_mean - max(params.stop_overflow, bo)) / bo
            if wl_ratio > threshold * 1.2:
                if overflow_ratio > threshold:
                    return True
                if overflow_range / overflow_mean < threshold:
                    return True
                if overflow_diff > 0.6:
                    return True
            return False

        def check_divergence(window=50, threshold=0.05):
            if len(divergence_list) < window or best["metric"] is None:
                return False
            xs = divergence_list[-window:]
            # plain floats decide every comparison that is not within rounding
            # of its bound; otherwise numpy's means (the reference's) decide
            ov = [p[1] for p in xs]
            n = len(ov)
            overflow_mean = sum(ov) / n
            wl_mean = sum(p[0] for p in xs) / n
            bh, bo = best["metric"].hpwl, best["metric"].overflow
            wl_ratio = (wl_mean - bh) / bh
            overflow_ratio = (overflow_mean - max(params.stop_overflow, bo)) / bo
            rng_ratio = (max(ov) - min(ov)) / overflow_mean if overflow_mean != 0.0 else None
            close = lambda a, b: abs(a - b) <= 1e-9 * max(abs(a), abs(b))  # noqa: E731
            if rng_ratio is None or close(wl_ratio, threshold * 1.2) or close(overflow_ratio, threshold) or \
                    close(rng_ratio, threshold):
                return divergence_numpy(xs, threshold)
            if wl_ratio > threshold * 1.2:
                if overflow_ratio > threshold:
                    return True
                if rng_ratio < threshold:
                    return True
                ups = sum(1 for a, b in zip(ov, ov[1:]) if b > a)
                if ups / (n - 1) > 0.6:
                    return True
            return False

        def check_plateau(x, window=10, threshold=0.001):
            if len(x) < window:
                return False
            x = x[-window:]
            # plain floats decide unless the ratio is within rounding of the
            # threshold, where numpy's mean (the reference's) decides
            total = sum(x)
            if total > 0.0:
                r = (max(x) - min(x)) / (total / window)
                if abs(r - threshold) > 1e-9 * threshold:
                    return r < threshold
            return (np.max(x) - np.min(x)) / np.mean(x) < threshold

        for Lgamma_step in range(start_step, model.Lgamma_iteration):
            if checkpoint_every and checkpoint_fn is not None and iteration > start_step and \
                    iteration % checkpoint_every == 0:
                checkpoint_fn(checkpoint())
            all_metrics.append([])
            llam = all_metrics[-1]
            for Llambda_step in range(model.Llambda_density_weight_iteration):
                llam.append([])
                lsub = llam[-1]
                for Lsub_step in range(model.Lsub_iteration):
                    if (params.stop_overflow * 1.1 < overflow_list[-1] < params.stop_overflow * 4
                            and check_divergence(50, overflow_list[-1])):
                        if hasattr(stepper, "best_position"):
                            stepper.best_position()  # completes a pending copy into best["pos"]
                        stepper.set_position(best["pos"])
                        stop_placement = True
                        self.divergence_iteration = iteration
                        logger.error("possible DIVERGENCE detected, roll back to the best position recorded")
                    t0 = time.time()
                    if hasattr(stepper, "step_gen"):
                        h, o, md, obj = yield from stepper.step_gen(iteration == 0)
                    else:
                        h, o, md, obj = stepper.step(iteration == 0)
                    cur = EvalMetrics(iteration, h, o, md, obj)
                    lsub.append(cur)
                    if best["metric"] is None or best["metric"].overflow > o:
                        best["metric"] = cur
                        if hasattr(stepper, "record_best"):
                            # copied on the device only before its slot is reused
                            best["pos"] = stepper.record_best(best["pos"])
                        elif best["pos"] is None:
                            best["pos"] = stepper.position().clone()
                        else:
                            best["pos"].copy_(stepper.position())
                    overflow_list.append(o)
                    divergence_list.append([h, o])
                    if iteration - last_perturb_iter > 50 and check_plateau(overflow_list, 15, 0.001):
                        if overflow_list[-1] > 0.9:  # stuck at high overflow
                            model.quad_penalty = True
                            model.density_factor *= 2
                            if overflow_list[-1] > 0.95:  # stuck at very high overflow
                                intensity = min(max(40 + (120 - 40) * (overflow_list[-1] - 0.95) * 10, 40), 90)
                                self._entropy_injection(stepper, design, 0.996, intensity, noise_gen)
                            last_perturb_iter = iteration
                    self.iteration_times.append(time.time() - t0)
                    if callback is not None:
                        callback(iteration, cur)
                    iteration += 1
                    if self._lsub_stop(model, lsub):
                        break
                flat_llambda += 1
                if flat_llambda > 1:
                    # RePlAce hpwl-mode density weight update (dreamplace/PlaceObj.py:840-851)
                    prev = llam[-2][-1] if len(llam) > 1 else all_metrics[-2][-1][-1]
                    delta = llam[-1][-1].hpwl - prev.hpwl
                    if delta < 0:
                        mu = upper * max(math.pow(0.9999, float(flat_llambda)), 0.98)
                    else:
                        mu = upper * min(max(math.pow(upper, -delta / ref_hpwl), lower), upper)
                    if not device_updates:
                        with torch.no_grad():
                            model.density_weight.mul_(mu)
                if self._llambda_stop(params, llam):
                    break
            # gamma = base * 10^((overflow - 0.1) * 20/9 - 1) (dreamplace/PlaceObj.py:901-915)
            coef = math.pow(10, (llam[-1][-1].overflow - 0.1) * 20 / 9 - 1)
            if not device_updates:
                with torch.no_grad():
                    model.gamma.fill_(base_gamma * coef)
            if self._lgamma_stop(params, design, Lgamma_step, all_metrics, best) or stop_placement:
                break
        if device_updates:
            stepper.sync_model()
        with torch.no_grad():
            self.pos[0].data.copy_(stepper.position())
        self.metrics = all_metrics
        self.best = best
        return all_metrics

    @staticmethod
    def _restore_model(model, resume):
        m = resume["model"]
        dev = model.density_weight.device
        model.density_factor = m["density_factor"]
        model.quad_penalty = m["quad_penalty"]
        model.density_weight = m["density_weight"].to(dev)
        model.gamma.data.copy_(m["gamma"].to(dev))
        if m["init_density"] is not None:
            model.init_density = m["init_density"].to(dev)
            model.density_weight_grad_precond = torch.where(model.init_density > 0, 1 / model.init_density,
                                                            model.init_density)
            model.quad_penalty_coeff = model.density_quad_coeff / 2 * model.density_weight_grad_precond

    @staticmethod
    def _entropy_injection(stepper, design, shrink_factor, noise_intensity, generator=None):
        """Shrink all nodes towards the movable cells' centroid and add Gaussian
        noise of ``noise_intensity`` layout units, fixed nodes kept in place
        (reference dreamplace/NonLinearPlace.py:572-606, "random" mode).  The
        perturbed position replaces v_k; the optimizer state is left as is, as
        in the reference, whose v_k is the position parameter itself."""
        d = design
        n, m, nf = d.num_nodes, d.num_movable_nodes, d.num_filler_nodes
        with torch.no_grad():
            pos = stepper.position().clone()
            xc = pos[:m].mean()
            yc = pos[n:n + m].mean()
            fixed_x = pos[m:n - nf].clone()
            fixed_y = pos[n + m:2 * n - nf].clone()
            if shrink_factor != 1:
                pos[:n] = (pos[:n] - xc) * shrink_factor + xc
                pos[n:] = (pos[n:] - yc) * shrink_factor + yc
            if noise_intensity > 0.01:
                pos.add_(noise_intensity * torch.randn(2 * n, device=pos.device, generator=generator))
            pos[m:n - nf] = fixed_x
            pos[n + m:2 * n - nf] = fixed_y
            stepper.set_position(pos)
        logger.info("entropy injection: shrink %g, noise intensity %g", shrink_factor, noise_intensity)

    @staticmethod
    def _lsub_stop(model, lsub):
        w = max(min(model.Lsub_iteration // 2, 3), 1)
        if len(lsub) >= 2 * w:
            cur = sum(lsub[-1 - i].objective for i in range(w)) / w
            prev = sum(lsub[-1 - w - i].objective for i in range(w)) / w
            return cur >= prev * 0.999
        return False

    @staticmethod
    def _llambda_stop(params, llam):
        if len(llam) > 1:
            cur, prev = llam[-1][-1], llam[-2][-1]
            return (cur.overflow < params.stop_overflow and cur.hpwl > prev.hpwl) or cur.max_density < 1.0
        return False

    @staticmethod
    def _lgamma_stop(params, design, step, metrics, best):
        if len(metrics) > 1:
            cur, prev = metrics[-1][-1][-1], metrics[-2][-1][-1]
            if step > 100 and ((cur.overflow < params.stop_overflow and cur.hpwl > prev.hpwl)
                               or cur.max_density < design.target_density):
                return True
        if len(metrics) > 50:
            cur, prev = metrics[-1][-1][-1], metrics[-50][-1][-1]
            if cur.overflow > prev.overflow and cur.hpwl > best["metric"].hpwl * 2:
                return True
        return False


def place(design, params=None, device=None, max_iterations=None, callback=None):
    """Runs global placement; returns (placer, final metrics as python floats)."""
    params = params or Params()
    placer = NonLinearPlace(params, design, device)
    metrics = placer(params, design, max_iterations=max_iterations, callback=callback)
    last = metrics[-1][-1][-1]
    return placer, {"iterations": last.iteration + 1, "hpwl": last.hpwl, "overflow": last.overflow,
                    "max_density": last.max_density}
