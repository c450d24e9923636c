"""CPU: the MLP oracle of the learned initialiser.

BF16 rounding is checked against torch's float32 -> bfloat16 conversion; the
rounding-free float64 gradients against central finite differences (h = 1e-6,
gate 1e-6 relative L2).
"""
import numpy as np
import torch

from oracle import mlp as om


def test_bf16_rounding_matches_torch():
    x = np.random.default_rng(0).normal(0, 3, 20000).astype(np.float32)
    x[:4] = [0.0, -0.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8]  # ties to even both ways
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(om.bf16(x), ref)


def test_gradients_match_finite_differences():
    D, H, O, M = 128, 128, 5, 6
    rng = np.random.default_rng(1)
    w = om.init_weights(D, H, O, seed=2).astype(np.float64)
    w += om.valid_mask(D, H, O) * rng.normal(0, 0.02, w.shape)
    X = rng.normal(0, 1, (M, D))
    T = rng.normal(0, 1, (M, O))
    wout = rng.uniform(0.5, 2.0, O)
    _, _, g = om.forward_backward(w, X, T, wout, D, H, O, rounding=False)
    idx = rng.choice(np.flatnonzero(om.valid_mask(D, H, O)), 60, replace=False)
    fd = []
    for i in idx:
        e = np.zeros_like(w)
        e[i] = 1e-6
        lp = om.forward_backward(w + e, X, T, wout, D, H, O, rounding=False)[0]
        lm = om.forward_backward(w - e, X, T, wout, D, H, O, rounding=False)[0]
        fd.append((lp - lm) / 2e-6)
    fd = np.array(fd)
    assert np.linalg.norm(g[idx] - fd) < 1e-6 * np.linalg.norm(fd)
    # the padding rows of W3 / b3 get no gradient
    assert np.all(g[~om.valid_mask(D, H, O)] == 0)
