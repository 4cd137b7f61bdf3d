"""Global placement driver.

Mirrors the reference's ``NonLinearPlace.__call__`` for the default flow
(dreamplace/NonLinearPlace.py:49-798): one stage, nesterov, the three nested
loops Lgamma / Llambda / Lsub with their stop criteria, per-iteration HPWL and
overflow evaluation (dreamplace/EvalMetrics.py:100-141), density-weight and
gamma updates, best-position tracking, divergence rollback and the plateau
rule that turns on the quadratic density penalty.  The per-iteration metrics
(HPWL and overflow, accumulated in fp64) are read back once per iteration.
"""
import logging
import time

import numpy as np
import torch
from torch import nn

from .nesterov import NesterovAcceleratedGradientOptimizer
from .params import Params
from .place_obj import PlaceDataCollection, PlaceObj, build_ops

logger = logging.getLogger(__name__)


class EvalMetrics(object):
    """Per-iteration metrics (reference dreamplace/EvalMetrics.py)."""

    def __init__(self, iteration=None, detailed_step=None):
        self.iteration = iteration
        self.detailed_step = detailed_step
        self.objective = None
        self.hpwl = None
        self.overflow = None
        self.max_density = None
        self.gamma = None
        self.density_weight = None

    def evaluate(self, design, ops, pos):
        with torch.no_grad():
            self.hpwl = ops.hpwl_f64_op(pos)[0]
            ovf = ops.density_overflow_op.overflow_f64(pos)
            self.overflow = (ovf[0] / design.total_movable_node_area).reshape(1)
            self.max_density = ovf[1].reshape(1)

    def host(self):
        """(hpwl, overflow, max_density) as python floats (one device read)."""
        v = torch.stack([self.hpwl.reshape(()), self.overflow.reshape(()), self.max_density.reshape(())]).cpu()
        self._host = (float(v[0]), float(v[1]), float(v[2]))
        return self._host

    def __str__(self):
        h = getattr(self, "_host", None)
        if h is None:
            return "iteration %s" % self.iteration
        return "iteration %4d, HPWL %.6E, Overflow %.6E, MaxDensity %.3E" % (self.iteration, h[0], h[1], h[2])


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

    def __call__(self, params=None, design=None, max_iterations=None, callback=None):
        params = params or self.params
        design = design or self.design
        torch.manual_seed(params.random_seed)
        gp = dict(params.global_place_stages[0])
        if max_iterations is not None:
            gp["iteration"] = max_iterations
        model = PlaceObj(0.0, params, design, self.data_collections, self.op_collections, gp).to(self.device)
        self.model = model
        pos = self.data_collections.pos[0]
        optimizer = NesterovAcceleratedGradientOptimizer(self.parameters(), lr=0.0,
                                                         obj_and_grad_fn=model.obj_and_grad_fn,
                                                         constraint_fn=self.op_collections.move_boundary_op)
        self.optimizer = optimizer
        if params.gp_noise_ratio > 0.0:
            model.ops.noise_op(pos, params.gp_noise_ratio)
        lr = model.estimate_initial_learning_rate(pos, gp["learning_rate"])
        for g in optimizer.param_groups:
            g["lr"] = lr.data
        all_metrics = []
        best = {"metric": None, "pos": None}
        overflow_list = [1.0]
        divergence_list = []
        last_perturb_iter = -50
        stop_placement = False
        iteration = 0
        self.iteration_times = []

        def check_divergence(window=50, threshold=0.05):
            if len(divergence_list) < window or best["metric"] is None:
                return False
            x = np.array(divergence_list[-window:])
            overflow_mean = np.mean(x[:, 1])
            overflow_diff = np.sum(np.maximum(0, np.sign(x[1:, 1] - x[:-1, 1]))) / (x.shape[0] - 1)
            overflow_range = np.max(x[:, 1]) - np.min(x[:, 1])
            wl_mean = np.mean(x[:, 0])
            bh, bo = best["metric"]._host[0], best["metric"]._host[1]
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

        def check_plateau(x, window=10, threshold=0.001):
            if len(x) < window:
                return False
            x = x[-window:]
            return (np.max(x) - np.min(x)) / np.mean(x) < threshold

        for Lgamma_step in range(model.Lgamma_iteration):
            all_metrics.append([])
            llam = all_metrics[-1]
            for Llambda_step in range(model.Llambda_density_weight_iteration):
                llam.append([])
                lsub = llam[-1]
                for Lsub_step in range(model.Lsub_iteration):
                    if (params.stop_overflow * 1.1 < overflow_list[-1] < params.stop_overflow * 4
                            and check_divergence(50, overflow_list[-1])):
                        self.pos[0].data.copy_(best["pos"])
                        stop_placement = True
                        logger.error("possible DIVERGENCE detected, roll back to the best position recorded")
                    t0 = time.time()
                    cur = EvalMetrics(iteration, (Lgamma_step, Llambda_step, Lsub_step))
                    lsub.append(cur)
                    self.op_collections.move_boundary_op(pos)
                    if float(model.density_weight.mean()) == 0.0:
                        model.initialize_density_weight(params, design)
                    optimizer.zero_grad(set_to_none=False)
                    cur.evaluate(design, self.op_collections, pos)
                    optimizer.step()
                    cur.gamma = model.gamma.data.clone()
                    cur.density_weight = model.density_weight.data.clone()
                    cur.objective = optimizer.param_groups[0]["obj_k_1"][0].data.clone()
                    h, o, md = cur.host()
                    if best["metric"] is None or best["metric"]._host[1] > o:
                        best["metric"] = cur
                        if best["pos"] is None:
                            best["pos"] = self.pos[0].data.clone()
                        else:
                            best["pos"].copy_(self.pos[0].data)
                    overflow_list.append(o)
                    divergence_list.append([h, o])
                    if iteration - last_perturb_iter > 50 and check_plateau(overflow_list, 15, 0.001):
                        if overflow_list[-1] > 0.9:
                            model.quad_penalty = True
                            model.density_factor *= 2
                            last_perturb_iter = iteration
                    self.iteration_times.append(time.time() - t0)
                    if callback is not None:
                        callback(iteration, cur)
                    iteration += 1
                    if self._lsub_stop(model, lsub):
                        break
                if Lgamma_step * model.Llambda_density_weight_iteration + Llambda_step + 1 > 1:
                    prev = llam[-2][-1] if len(llam) > 1 else all_metrics[-2][-1][-1]
                    model.ops.update_density_weight_op(llam[-1][-1], prev, Lgamma_step + 1)
                if self._llambda_stop(params, llam):
                    break
            model.ops.update_gamma_op(Lgamma_step, llam[-1][-1].overflow)
            if self._lgamma_stop(params, design, Lgamma_step, all_metrics, best) or stop_placement:
                break
        self.metrics = all_metrics
        self.best = best
        return all_metrics

    @staticmethod
    def _lsub_stop(model, lsub):
        w = max(min(model.Lsub_iteration // 2, 3), 1)
        if len(lsub) >= 2 * w:
            cur = sum(float(lsub[-1 - i].objective) for i in range(w)) / w
            prev = sum(float(lsub[-1 - w - i].objective) for i in range(w)) / w
            return cur >= prev * 0.999
        return False

    @staticmethod
    def _llambda_stop(params, llam):
        if len(llam) > 1:
            cur, prev = llam[-1][-1]._host, llam[-2][-1]._host
            return (cur[1] < params.stop_overflow and cur[0] > prev[0]) or cur[2] < 1.0
        return False

    @staticmethod
    def _lgamma_stop(params, design, step, metrics, best):
        if len(metrics) > 1:
            cur, prev = metrics[-1][-1][-1]._host, metrics[-2][-1][-1]._host
            if step > 100 and ((cur[1] < params.stop_overflow and cur[0] > prev[0])
                               or cur[2] < design.target_density):
                return True
        if len(metrics) > 50:
            cur, prev = metrics[-1][-1][-1]._host, metrics[-50][-1][-1]._host
            if cur[1] > prev[1] and cur[0] > best["metric"]._host[0] * 2:
                return True
        return False


def place(design, params=None, device=None, max_iterations=None, callback=None):
    """Runs global placement; returns (placer, final metrics as python floats)."""
    params = params or Params()
    placer = NonLinearPlace(params, design, device)
    metrics = placer(params, design, max_iterations=max_iterations, callback=callback)
    last = metrics[-1][-1][-1]
    return placer, {"iterations": last.iteration + 1, "hpwl": last._host[0], "overflow": last._host[1],
                    "max_density": last._host[2]}
