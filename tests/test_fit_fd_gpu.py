"""GPU: the fused fit gradient against central finite differences at the c2 adjoint size.

512x512 grayscale, 2048 Gaussians, 2 planes (FFT grid 1664 x 1664 = (2^7 13)^2).
One fused step with every learning rate at 0, noise off and no clipping leaves
the parameters unchanged and the raw dL/d(params) in the gradient buffer. For
each of the 9 raw parameter kinds, the noise-free loss of cvqpg_fit_evaluate is
differenced along 4 random +-1 directions over 64 Gaussians (directional
derivatives: the loss change of a single parameter is below the float32
resolution of the loss itself); gate 3e-2 relative L2 per kind.

Memory case (3840 x 2160, 200k Gaussians, one channel, splat adjoint only):
the render forward + adjoint fit in a few GB and the adjoint is linear in dL/dU.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

RAW = ("means_2d", "pre_act_scales", "pre_act_rotation", "colours", "pre_act_phase", "pre_act_opacities",
       "curvature")


def test_fused_gradient_matches_finite_differences_512():
    from complex_valued_quadratic_phase_gaussian_b200 import scenes
    from complex_valued_quadratic_phase_gaussian_b200.fit import FitConfig, Fitter, synthetic_init
    H = W = 512
    img, depth = scenes.grayscale_blobs(H, W, seed=2)
    targets, q = scenes.multiplane_targets_device(img, depth, 2)
    cfg = FitConfig(img_size=(W, H), num_gaussians=2048, wavelengths=[515e-9], pixel_pitch=8e-6, num_planes=2,
                    d_val=1.5e-3, volume_depth=1e-3, group_lrs=[0.0] * 6, cosine_means=False, inject_noise=False,
                    warmup_iters=0, num_itrs=10, seed=4)
    assert cfg.resolved_pad() == [832, 832]
    f = Fitter(cfg, targets, q, init=synthetic_init(cfg, 4))
    f.params.max_grad_norm = 1e30
    before = f.flat.clone()
    f.step()
    torch.cuda.synchronize()
    assert torch.equal(f.flat, before)  # lr 0: nothing moved
    grads = f.grads.clone()
    rng = np.random.default_rng(0)
    gids = rng.choice(2048, 64, replace=False)
    N = 2048
    # (flat offset of kind k for Gaussian g) and step; one FD per random +-1 direction over the 64 Gaussians
    kinds = {"mean_x": (0, 2, 1e-3), "mean_y": (1, 2, 1e-3), "scale_x": (2 * N, 2, 1e-2), "scale_y": (2 * N + 1, 2, 1e-2),
             "rotation": (4 * N, 1, 1e-2), "colour": (5 * N, 1, 1e-2), "phase": (6 * N, 1, 1e-2),
             "opacity": (7 * N, 1, 1e-2), "curvature": (8 * N, 1, 1e-2)}
    for name, (base, stride, h) in kinds.items():
        idx = torch.from_numpy(base + stride * gids).cuda()
        an, fd = [], []
        for _ in range(4):
            d = torch.from_numpy(rng.choice([-1.0, 1.0], 64).astype(np.float32)).cuda()
            f.flat[idx] = before[idx] + h * d
            lp = f.evaluate()["loss"]
            f.flat[idx] = before[idx] - h * d
            lm = f.evaluate()["loss"]
            f.flat[idx] = before[idx]
            fd.append((lp - lm) / (2 * h))
            an.append(float((grads[idx].double() * d.double()).sum()))
        an, fd = np.array(an), np.array(fd)
        err = np.linalg.norm(an - fd) / np.linalg.norm(fd)
        assert err < 3e-2, (name, err, an, fd)


def test_splat_adjoint_memory_4k():
    from complex_valued_quadratic_phase_gaussian_b200.rasterizer import render_backward, render_forward
    n, W, H = 200_000, 3840, 2160
    rng = np.random.default_rng(1)
    torch.cuda.reset_peak_memory_stats()
    means = torch.from_numpy(np.stack([rng.uniform(0, W, n), rng.uniform(0, H, n)], 1).astype(np.float32)).cuda()
    inv = torch.tensor([0.22, 0.01, 0.2], device="cuda").repeat(n, 1)
    col = torch.rand(n, 1, device="cuda")
    ph = torch.rand(n, 1, device="cuda") * 6.28
    z = torch.rand(n, device="cuda")
    radii = torch.full((n,), 12, dtype=torch.int32, device="cuda")
    k = torch.tensor([2 * np.pi / 515e-9], dtype=torch.float32, device="cuda")
    args = (means, inv, col, ph, z, z * 300, z + 4, k)
    out, pl, ranges = render_forward(*args, 3.74e-6 ** 2, W, H, radii=radii)
    g = torch.polar(torch.rand(1, H, W, device="cuda"), torch.rand(1, H, W, device="cuda") * 6.28)
    d1 = render_backward(g, *args, pl, ranges, 3.74e-6 ** 2, W, H)
    d2 = render_backward(2 * g, *args, pl, ranges, 3.74e-6 ** 2, W, H)
    torch.cuda.synchronize()
    peak = torch.cuda.max_memory_allocated() / 2 ** 30
    assert peak < 4.0, peak
    for a, b in zip(d1, d2):
        assert torch.isfinite(a).all()
        assert torch.allclose(b, 2 * a, rtol=1e-4, atol=1e-6 * float(a.abs().max()))
