"""ePlace Nesterov optimizer with Lipschitz backtracking.

Mirrors ``NesterovAcceleratedGradientOptimizer.step_nobb`` of the reference
(dreamplace/NesterovAcceleratedGradientOptimizer.py:65-166): state u_k, v_k,
g_k, a_k, alpha_k, v_k_1, g_k_1; per step

    a_{k+1} = (1 + sqrt(4 a_k^2 + 1)) / 2,   coef = (a_k - 1) / a_{k+1}
    repeat (<= 10): u = v_k - alpha_k g_k;  v = u + coef (u - u_k);  constraint(v)
                    f, g = obj_and_grad(v);  alpha = |v - v_k| / |g - g_k|
                    accept when alpha > 0.95 alpha_k (alpha_k <- alpha either way)

The step-size estimate alpha (the two norms and their ratio) is computed in
fp64 on the device; the accept test is the only host read per trial.
"""
import torch
from torch.optim.optimizer import Optimizer


def _sqnorm_diff_f64(a, b):
    d = (a - b).to(torch.float64)
    return torch.dot(d, d)


class NesterovAcceleratedGradientOptimizer(Optimizer):
    def __init__(self, params, lr=0.0, obj_and_grad_fn=None, constraint_fn=None, use_bb=False):
        if lr < 0.0:
            raise ValueError("Invalid learning rate: {}".format(lr))
        defaults = dict(lr=lr, u_k=[], v_k=[], g_k=[], obj_k=[], a_k=[], alpha_k=[], v_k_1=[], g_k_1=[],
                        obj_k_1=[], v_kp1=[None], obj_eval_count=0)
        super().__init__(params, defaults)
        self.obj_and_grad_fn = obj_and_grad_fn
        self.constraint_fn = constraint_fn
        self.use_bb = use_bb
        if len(self.param_groups) != 1:
            raise ValueError("Only parameters with single tensor is supported")
        self.backtrack_counts = []

    def step(self, closure=None):
        if self.use_bb:
            raise NotImplementedError("the Barzilai-Borwein variant is not part of dreamplace_b200")
        return self.step_nobb(closure)

    def step_nobb(self, closure=None):
        loss = closure() if closure is not None else None
        group = self.param_groups[0]
        f_and_g = self.obj_and_grad_fn
        for i, p in enumerate(group['params']):
            if p.grad is None:
                continue
            if not group['u_k']:
                group['u_k'].append(p.data.clone())
                group['v_k'].append(p)
                obj, grad = f_and_g(group['v_k'][i])
                group['g_k'].append(grad.data.clone())
                group['obj_k'].append(obj.data.clone())
            u_k, v_k, g_k, obj_k = group['u_k'][i], group['v_k'][i], group['g_k'][i], group['obj_k'][i]
            if not group['a_k']:
                group['a_k'].append(torch.ones(1, dtype=torch.float64, device=g_k.device))
                group['v_k_1'].append(torch.zeros_like(v_k).requires_grad_(True))
                group['v_k_1'][i].data.copy_(group['v_k'][i] - group['lr'] * g_k)
                obj, grad = f_and_g(group['v_k_1'][i])
                group['g_k_1'].append(grad.data.clone())
                group['obj_k_1'].append(obj.data.clone())
            a_k, v_k_1, g_k_1, obj_k_1 = group['a_k'][i], group['v_k_1'][i], group['g_k_1'][i], group['obj_k_1'][i]
            if not group['alpha_k']:
                group['alpha_k'].append((_sqnorm_diff_f64(v_k.data, v_k_1.data) /
                                         _sqnorm_diff_f64(g_k, g_k_1)).sqrt().reshape(1))
            alpha_k = group['alpha_k'][i]
            if group['v_kp1'][i] is None:
                group['v_kp1'][i] = torch.zeros_like(v_k).requires_grad_(True)
            v_kp1 = group['v_kp1'][i]
            a_kp1 = (1 + (4 * a_k.pow(2) + 1).sqrt()) / 2
            coef = ((a_k - 1) / a_kp1).to(torch.float32)
            backtrack = 0
            while True:
                step = alpha_k.to(torch.float32)
                u_kp1 = v_k.data - step * g_k
                v_kp1.data.copy_(u_kp1 + coef * (u_kp1 - u_k))
                if self.constraint_fn is not None:
                    self.constraint_fn(v_kp1)
                f_kp1, g_kp1 = f_and_g(v_kp1)
                alpha_kp1 = (_sqnorm_diff_f64(v_kp1.data, v_k.data) / _sqnorm_diff_f64(g_kp1.data, g_k)).sqrt()
                backtrack += 1
                group['obj_eval_count'] += 1
                accept = bool((alpha_kp1 > 0.95 * alpha_k).item())
                alpha_k.copy_(alpha_kp1)
                if accept or backtrack >= 10:
                    break
            self.backtrack_counts.append(backtrack)
            v_k_1.data.copy_(v_k.data)
            g_k_1.data.copy_(g_k.data)
            obj_k_1.data.copy_(obj_k.data)
            u_k.data.copy_(u_kp1)
            v_k.data.copy_(v_kp1.data)
            g_k.data.copy_(g_kp1.data)
            obj_k.data.copy_(f_kp1.data)
            a_k.data.copy_(a_kp1)
        return loss
