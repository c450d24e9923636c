"""GPU: the fused multi-plane loss (cvqpg_loss_forward_backward) against the float64 oracle.

Gates: total and per-plane loss within 1e-5 relative, per-plane MSE within
1e-5 relative, SSIM within 1e-5 absolute (float32 moments; an 11x11 image has one map position per channel), dL/d(pred) within 1e-4 relative L2.
The noisy-target terms use the same Philox4x32-10 + Box-Muller stream in the
kernel and in the oracle, so the noisy loss is compared directly.
"""
import ctypes

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import loss as oloss

pytestmark = pytest.mark.gpu


def _case(P, C, H, W, seed):
    rng = np.random.default_rng(seed)
    pred = np.clip(rng.uniform(-0.1, 1.2, (P, C, H, W)), 0, 1).astype(np.float32)
    targets = rng.uniform(0, 1, (P, C, H, W)).astype(np.float32)
    # smooth structure so SSIM is far from 0 and its gradient is not noise-dominated
    yy, xx = np.mgrid[0:H, 0:W]
    base = 0.5 + 0.4 * np.sin(xx / 7.0) * np.cos(yy / 5.0)
    targets = (0.7 * base[None, None] + 0.3 * targets).astype(np.float32)
    pred = np.clip(0.8 * targets + 0.25 * pred - 0.02, 0, 1).astype(np.float32)
    depth = rng.integers(0, P, (H, W)).astype(np.uint8)
    return pred, targets, depth


@pytest.mark.parametrize("P,C,H,W,noise,it", [(3, 3, 45, 70, True, 7), (1, 1, 256, 256, False, 0),
                                              (8, 1, 24, 40, True, 3), (2, 3, 11, 11, True, 1),
                                              (3, 1, 97, 161, True, 123456)])
def test_loss_matches_oracle(P, C, H, W, noise, it):
    from complex_valued_quadratic_phase_gaussian_b200.loss import MultiplaneLoss
    pred, targets, depth = _case(P, C, H, W, seed=P * 1000 + H)
    seed = 0x1234_5678_9ABC
    lf = MultiplaneLoss(torch.from_numpy(targets).cuda(), torch.from_numpy(depth).cuda(), inject_noise=noise,
                        seed=seed)
    out, g = lf(torch.from_numpy(pred).cuda(), iteration=it)
    torch.cuda.synchronize()
    out, g = out.cpu().numpy().astype(np.float64), g.cpu().numpy()
    z = oloss.plane_noise((P, C, H, W), seed, it) if noise else None
    total, mses, ssims, losses, gx = oloss.multiplane_loss_pred(pred, targets, depth, noise=z)
    assert abs(out[0] - total) < 1e-5 * abs(total)
    np.testing.assert_allclose(out[1:1 + P], mses, rtol=1e-5)
    np.testing.assert_allclose(out[1 + P:1 + 2 * P], ssims, atol=1e-5)
    np.testing.assert_allclose(out[1 + 2 * P:1 + 3 * P], losses, rtol=1e-5)
    assert rel_l2(g, gx) < 1e-4, rel_l2(g, gx)


def test_loss_is_deterministic_and_noise_follows_iteration():
    from complex_valued_quadratic_phase_gaussian_b200.loss import MultiplaneLoss
    pred, targets, depth = _case(3, 3, 64, 96, seed=5)
    lf = MultiplaneLoss(torch.from_numpy(targets).cuda(), torch.from_numpy(depth).cuda(), seed=9)
    x = torch.from_numpy(pred).cuda()
    a_out, a_g = lf(x, iteration=4)
    b_out, b_g = lf(x, iteration=4)
    c_out, c_g = lf(x, iteration=5)
    torch.cuda.synchronize()
    assert torch.equal(a_out, b_out) and torch.equal(a_g, b_g)
    assert not torch.equal(a_g, c_g)


def test_loss_rejects_bad_parameters():
    from complex_valued_quadratic_phase_gaussian_b200 import _lib
    from complex_valued_quadratic_phase_gaussian_b200.loss import LossParams
    lib = _lib.lib()
    sz = ctypes.c_size_t(0)
    assert lib.cvqpg_loss_workspace_size(ctypes.byref(LossParams(3, 3, 10, 64, 1, 1, 1, 0.005, 1e-3, 1, 0)),
                                         ctypes.byref(sz)) == 5  # SSIM window does not fit
    assert lib.cvqpg_loss_workspace_size(ctypes.byref(LossParams(3, 9, 64, 64, 1, 1, 1, 0.005, 1e-3, 1, 0)),
                                         ctypes.byref(sz)) == 5  # more planes than supported
    assert lib.cvqpg_loss_workspace_size(ctypes.byref(LossParams(2, 3, 64, 64, 1, 1, 1, 0.005, 1e-3, 1, 0)),
                                         ctypes.byref(sz)) == 2  # channels


@pytest.mark.parametrize("P,C,H,W", [(3, 3, 45, 70), (1, 1, 256, 256), (2, 3, 11, 11), (3, 1, 97, 161)])
def test_target_moments_path_matches_on_the_fly(P, C, H, W):
    """Precomputed target moments (cvqpg_loss_target_moments) against filtering the targets in the
    loss call: same window, same fma order, so the results agree to float32 rounding (1e-6)."""
    from complex_valued_quadratic_phase_gaussian_b200.loss import MultiplaneLoss
    pred, targets, depth = _case(P, C, H, W, seed=77 + H)
    t, d = torch.from_numpy(targets).cuda(), torch.from_numpy(depth).cuda()
    a = MultiplaneLoss(t, d, seed=3, target_moments=True)
    b = MultiplaneLoss(t, d, seed=3, target_moments=False)
    assert a.moments is not None and b.moments is None
    x = torch.from_numpy(pred).cuda()
    oa, ga = a(x, iteration=11)
    ob, gb = b(x, iteration=11)
    torch.cuda.synchronize()
    assert torch.allclose(oa, ob, rtol=1e-6, atol=0)
    assert rel_l2(ga.cpu().numpy(), gb.cpu().numpy()) < 1e-6


def test_target_moments_against_float64_window():
    """cvqpg_loss_target_moments: (mu_T, E_w[T^2]) on the valid map, against a float64 11x11 window."""
    from complex_valued_quadratic_phase_gaussian_b200.loss import MultiplaneLoss
    P, C, H, W = 2, 3, 50, 77
    _, targets, depth = _case(P, C, H, W, seed=12)
    lf = MultiplaneLoss(torch.from_numpy(targets).cuda(), torch.from_numpy(depth).cuda())
    torch.cuda.synchronize()
    mom = lf.moments.view(P * C, H - 10, W - 10, 2).cpu().numpy().astype(np.float64)
    g = np.exp(-((np.arange(11) - 5.0) ** 2) / (2 * 1.5 ** 2))
    g /= g.sum()
    w2 = np.outer(g, g)
    T = targets.reshape(P * C, H, W).astype(np.float64)
    mu = np.zeros((P * C, H - 10, W - 10))
    e2 = np.zeros_like(mu)
    for a in range(11):
        for b in range(11):
            win = T[:, a:a + H - 10, b:b + W - 10]
            mu += w2[a, b] * win
            e2 += w2[a, b] * win * win
    np.testing.assert_allclose(mom[..., 0], mu, atol=2e-6)
    np.testing.assert_allclose(mom[..., 1], e2, atol=2e-6)
