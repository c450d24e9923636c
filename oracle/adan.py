"""Oracle: Adan optimiser and clip_grad_norm_ (numpy float64). Test infrastructure only.

Restates utils/optimizer.py:104-262 (Adan.step with foreach=False, i.e.
_single_tensor_adan) including the per-group step counter that advances even
for a group without gradients (optimizer.py:146-149 run before the
params_with_grad check at :176), and torch.nn.utils.clip_grad_norm_ as used at
train_2d_gaussian_rgb.py:209 (total norm over tensors that have gradients,
coefficient max_norm / (norm + 1e-6) clamped to 1).
"""
import numpy as np


def clip_grad_norm(grads, max_norm):
    """grads: list of arrays or None. Scales in place-equivalent; returns (new grads, total norm)."""
    present = [g for g in grads if g is not None]
    total = float(np.sqrt(sum(float((g.astype(np.float64) ** 2).sum()) for g in present)))
    coef = min(max_norm / (total + 1e-6), 1.0)
    return [None if g is None else g * coef for g in grads], total


class Adan:
    def __init__(self, groups, betas=(0.98, 0.92, 0.99), eps=1e-8, weight_decay=0.0, no_prox=False):
        """groups: list of dicts {'params': [names], 'lr': float}."""
        self.groups = [dict(g) for g in groups]
        self.betas, self.eps, self.wd, self.no_prox = betas, eps, weight_decay, no_prox
        self.state = {}

    def step(self, params, grads):
        """params/grads: dicts name -> array (grad None = no gradient). Updates params in place."""
        b1, b2, b3 = self.betas
        for g in self.groups:
            g["step"] = g.get("step", 0) + 1
            step = g["step"]
            bc1, bc2, bc3 = 1 - b1 ** step, 1 - b2 ** step, 1 - b3 ** step
            lr = g["lr"]
            for name in g["params"]:
                grad = grads.get(name)
                if grad is None:
                    continue
                grad = np.asarray(grad, dtype=np.float64)
                st = self.state.setdefault(name, {})
                if not st:
                    st["exp_avg"] = np.zeros_like(grad)
                    st["exp_avg_sq"] = np.zeros_like(grad)
                    st["exp_avg_diff"] = np.zeros_like(grad)
                if "neg_pre_grad" not in st or step == 1:
                    st["neg_pre_grad"] = -grad.copy()
                ng = st["neg_pre_grad"] + grad
                st["exp_avg"] = st["exp_avg"] * b1 + (1 - b1) * grad
                st["exp_avg_diff"] = st["exp_avg_diff"] * b2 + (1 - b2) * ng
                ng = ng * b2 + grad
                st["exp_avg_sq"] = st["exp_avg_sq"] * b3 + (1 - b3) * ng * ng
                denom = np.sqrt(st["exp_avg_sq"]) / np.sqrt(bc3) + self.eps
                p = params[name]
                if self.no_prox:
                    p *= 1 - lr * self.wd
                    p -= lr / bc1 * st["exp_avg"] / denom
                    p -= lr * b2 / bc2 * st["exp_avg_diff"] / denom
                else:
                    p -= lr / bc1 * st["exp_avg"] / denom
                    p -= lr * b2 / bc2 * st["exp_avg_diff"] / denom
                    p /= 1 + lr * self.wd
                st["neg_pre_grad"] = -grad
