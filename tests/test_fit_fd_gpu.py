"""GPU: the fused fit gradient against FP64 central finite differences and against the
reference's autograd, at the adjoint-check size: 512x512 grayscale, 2048 Gaussians, 2 planes
(FFT grid 1664 x 1664 = (2^7 13)^2).

One fused step with noise off and no clipping leaves the raw dL/d(params) (after nan_to_num)
in the gradient buffer. For 64 random Gaussians x all 9 raw parameters, the noise-free loss is
differenced in float64 by oracle/fd64.py (the oracle's loss, one Gaussian moved at a time, its
tile lists held fixed and the replicate guard band held at its base value, as the reference's
no_grad band is), with central differences at h = 1e-3 and the Richardson combination of
h = 1e-3 and 5e-4 (which removes the h^2 truncation term: at h = 1e-3 a raw mean moves
0.26 px, a tenth of a Gaussian's width). Gate: per parameter kind, the median relative error of
the Richardson differences <= 1e-3; the worst case and the plain h = 1e-3 figures are printed.

The full gradient is also compared with the reference's own autograd on the same scene: the
reference CUDA rasterizer (oracle/_ref) under the torch propagator and loss of the reference loop
(oracle/torch_port.py, pinned to the reference loop's goldens), float32: <= 1e-3 relative L2 per
tensor over the Gaussians whose reference gradient is finite. The others are a float32 quirk of
the reference on the GPU: its amplitude clamp goes through torch.angle and torch.abs
(train_2d_gaussian_rgb.py:91-93), and angle's backward divides by |U|^2, which underflows to 0
where only Gaussian tails clamped at exp(-50) reach a pixel; the NaN it makes there reaches every
Gaussian whose tile list holds that pixel, and nan_to_num (train_2d_gaussian_rgb.py:206-208) zeroes
their whole gradient. The fused adjoint of the clamp has no such division (it is the identity for
|U| <= 1) and matches the FP64 differences above. The test checks that the excluded Gaussians are
exactly those with a non-finite reference gradient and that they are a minority.

Memory case (3840 x 2160, 200k Gaussians, one channel, splat adjoint only):
the render forward + adjoint fit in a few GB and the adjoint is linear in dL/dU.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

RAW = ("means_2d", "pre_act_scales", "pre_act_rotation", "colours", "pre_act_phase", "pre_act_opacities",
       "curvature")


@pytest.fixture(scope="module")
def c2_fit():
    from complex_valued_quadratic_phase_gaussian_b200 import scenes
    from complex_valued_quadratic_phase_gaussian_b200.fit import FitConfig, Fitter, synthetic_init
    H = W = 512
    img, depth = scenes.grayscale_blobs(H, W, seed=2)
    targets, q = scenes.multiplane_targets_device(img, depth, 2)
    cfg = FitConfig(img_size=(W, H), num_gaussians=2048, wavelengths=[515e-9], pixel_pitch=8e-6, num_planes=2,
                    d_val=1.5e-3, volume_depth=1e-3, inject_noise=False, max_grad_norm=0.0, warmup_iters=0,
                    num_itrs=10, seed=4)
    assert cfg.resolved_pad() == [832, 832]
    init = synthetic_init(cfg, 4)
    f = Fitter(cfg, targets, q, init=init)
    f.step()
    torch.cuda.synchronize()
    grads = {k: f.grad(k).detach().cpu().numpy().astype(np.float64) for k in RAW}
    loss = f.history_records(last=1)[0][1]
    return dict(cfg=cfg, init={k: v.numpy() for k, v in init.items()}, targets=targets.cpu().numpy(),
                q=q.cpu().numpy(), grads=grads, loss=loss)


def test_fused_gradient_matches_fp64_central_differences_512(c2_fit):
    from oracle.fd64 import FiniteDifferenceLoss
    cfg = c2_fit["cfg"]
    fd = FiniteDifferenceLoss({k: v.astype(np.float64) for k, v in c2_fit["init"].items()}, cfg.W, cfg.H,
                              cfg.wavelengths, cfg.pixel_pitch, cfg.resolved_pad(), cfg.distances(),
                              cfg.resolved_aperture(), c2_fit["targets"], c2_fit["q"], device="cuda")
    assert abs(fd.base_loss() - c2_fit["loss"]) < 1e-5 * fd.base_loss()
    rng = np.random.default_rng(0)
    gids = rng.choice(cfg.num_gaussians, 64, replace=False)
    kinds = [("means_2d", 0), ("means_2d", 1), ("pre_act_scales", 0), ("pre_act_scales", 1), ("pre_act_rotation", None),
             ("colours", 0), ("pre_act_phase", 0), ("pre_act_opacities", None), ("curvature", None)]
    report = {}
    for key, idx in kinds:
        rich, plain, ours = [], [], []
        for g in gids:
            d1 = fd.central_difference(int(g), key, idx, h=1e-3)
            d2 = fd.central_difference(int(g), key, idx, h=5e-4)
            rich.append((4.0 * d2 - d1) / 3.0)
            plain.append(d1)
            ours.append(c2_fit["grads"][key][g] if idx is None else c2_fit["grads"][key][g, idx])
        rich, plain, ours = np.array(rich), np.array(plain), np.array(ours)
        err = np.abs(ours - rich) / np.maximum(np.abs(rich), 1e-300)
        err_plain = np.abs(ours - plain) / np.maximum(np.abs(plain), 1e-300)
        name = key if idx is None else f"{key}[{idx}]"
        report[name] = (float(np.median(err)), float(err.max()), float(np.median(err_plain)), rel_l2(ours, rich))
    for name, (med, worst, med_plain, agg) in report.items():
        print(f"FD64 {name}: median rel err {med:.2e} (worst {worst:.2e}); plain h=1e-3 median {med_plain:.2e}; "
              f"rel-L2 over the 64 {agg:.2e}")
    for name, (med, worst, med_plain, agg) in report.items():
        assert med <= 1e-3, (name, med, worst)
        assert agg <= 1e-3, (name, agg)


def test_fused_gradient_matches_reference_autograd_512(c2_fit):
    from oracle.torch_port import ReferencePipeline, load_reference_extension
    ext = load_reference_extension()
    if ext is None:
        pytest.skip("reference extension not built (oracle/build_ref.py needs the reference sources)")
    cfg = c2_fit["cfg"]
    P, C, H, W = cfg.num_planes, 1, cfg.H, cfg.W
    pipe = ReferencePipeline(c2_fit["init"], (W, H), cfg.wavelengths, cfg.pixel_pitch, cfg.resolved_pad(),
                             cfg.distances(), cfg.resolved_aperture(), c2_fit["targets"], c2_fit["q"],
                             renderer="cuda", warmup_iters=0, num_itrs=10, device="cuda", ext=ext,
                             noise=lambda it: np.zeros((P, C, H, W), np.float32))
    loss, raw_ref = pipe.gradients(sanitize=False)
    assert abs(loss - c2_fit["loss"]) < 1e-5 * loss
    n = cfg.num_gaussians
    finite = np.ones(n, bool)
    for k in RAW:
        finite &= np.isfinite(raw_ref[k].cpu().numpy()).reshape(n, -1).all(axis=1)
    print(f"reference autograd: {n - finite.sum()} of {n} Gaussians with a non-finite gradient (zeroed there)")
    assert finite.mean() > 0.5
    for k in RAW:
        ref = raw_ref[k].cpu().numpy().astype(np.float64)
        e = rel_l2(c2_fit["grads"][k][finite], ref[finite])
        print(f"reference autograd {k}: rel-L2 {e:.2e} over the {finite.sum()} Gaussians with finite gradients")
        assert e < 1e-3, (k, e)


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
