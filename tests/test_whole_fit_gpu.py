"""GPU: a whole fit, not single iterations. From the bench's start (1920x1080 RGB, 96,000
random-init Gaussians, 3 planes; and the 256x256 gray c0 case, 4096 Gaussians, 3 planes; seed 0),
2000 iterations of the fused fit (graph replays) and 2000 iterations of the reference loop on the
same GPU: its own CUDA rasterizer (compiled from its sources, oracle/_ref) under the torch
propagator, loss + SSIM and Adan of train_2d_gaussian_rgb.py:147-262 (oracle/torch_port.py,
pinned to the loop goldens). At 256x256 the reference loop is fed the fused fit's own
counter-based target noise (the oracle's restatement of the generator); at 1080p, where that
restatement is too slow on the host, it draws its own noise (torch.randn_like,
utils/propagator.py:432) from a seeded generator. The trajectories are never re-synchronised, so
the gates are on outcomes: the noise-free per-plane PSNR of both final
parameter sets, evaluated by the same kernel, within `db`, and the two loss curves within `loss`
(relative) at iterations 250, 1000 and 2000. Both loops sum gradients with float atomics, so
neither run repeats bit for bit, and the gates sit at about twice the reference loop's own
spread across repeated runs, measured on this B200: at 1080p its final PSNR moved by 0.03 dB; at
256x256 with 4096 Gaussians its final plane-3 PSNR ranged 32.58-32.81 dB over four runs (two of
them on identical noise) and its loss at iteration 2000 0.00267-0.00280. The 1080p reference loop
takes about two minutes here.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
RAW = ("means_2d", "pre_act_scales", "pre_act_rotation", "colours", "pre_act_phase", "pre_act_opacities",
       "curvature")
CASES = {
    "rgb1080": dict(W=1920, H=1080, N=96000, P=3, wl=[639e-9, 515e-9, 473e-9], pitch=3.74e-6, d_val=1e-3,
                    same_noise=False, db=0.2, loss=0.03),
    "gray256": dict(W=256, H=256, N=4096, P=3, wl=[515e-9], pitch=8e-6, d_val=1.5e-3, same_noise=True, db=0.5,
                    loss=0.08),
}
ITERS = 2000
CHECK = (250, 1000, 2000)


@pytest.mark.parametrize("case", sorted(CASES))
def test_whole_fit_reaches_the_reference_loops_psnr(case):
    from complex_valued_quadratic_phase_gaussian_b200 import scenes
    from complex_valued_quadratic_phase_gaussian_b200.fit import FitConfig, Fitter, synthetic_init
    from oracle import loss as oloss
    from oracle.torch_port import ReferencePipeline, load_reference_extension
    ext = load_reference_extension()
    if ext is None:
        pytest.skip("reference extension not built (oracle/build_ref.py needs the reference sources)")
    c = CASES[case]
    W, H, P = c["W"], c["H"], c["P"]
    img, depth = (scenes.rgb_blobs(H, W, seed=0) if len(c["wl"]) == 3 else scenes.grayscale_blobs(H, W, seed=0))
    targets, q = scenes.multiplane_targets_device(img, depth, P, device="cuda")
    cfg = FitConfig(img_size=(W, H), num_gaussians=c["N"], wavelengths=list(c["wl"]), pixel_pitch=c["pitch"],
                    num_planes=P, d_val=c["d_val"], volume_depth=1e-3, warmup_iters=400, num_itrs=ITERS, seed=0)
    init = synthetic_init(cfg, 0)

    f = Fitter(cfg, targets, q, init=init)
    f.capture()
    ours, done = {}, 0
    for it in CHECK:
        f.run(it - done)
        done = it
        ours[it] = f.history_records(last=1)[0][1]
    ours_eval = f.evaluate()

    C = len(c["wl"])
    noise = (lambda it: oloss.plane_noise((P, C, H, W), cfg.seed, it)) if c["same_noise"] else None
    torch.manual_seed(0)
    pipe = ReferencePipeline({k: v.numpy() for k, v in init.items()}, (cfg.W, cfg.H), cfg.wavelengths,
                             cfg.pixel_pitch, cfg.resolved_pad(), cfg.distances(), cfg.resolved_aperture(), targets,
                             q, renderer="cuda", warmup_iters=cfg.warmup_iters, num_itrs=cfg.num_itrs, device="cuda",
                             ext=ext, noise=noise)
    ref = {}
    for it in range(1, ITERS + 1):
        pipe.step()
        if it in CHECK:
            ref[it] = pipe.last_loss
    f.load_raw({k: pipe.params[k].detach() for k in RAW})
    ref_eval = f.evaluate()

    print(f"whole fit {case}, loss (ours / reference):", {it: (round(ours[it], 6), round(ref[it], 6)) for it in CHECK})
    print(f"whole fit {case}, final PSNR per plane: ours", np.round(ours_eval["psnr"], 3), "reference",
          np.round(ref_eval["psnr"], 3))
    assert np.all(np.isfinite(ours_eval["psnr"])) and np.all(np.isfinite(ref_eval["psnr"]))
    for it in CHECK:
        assert abs(ours[it] - ref[it]) <= c["loss"] * ref[it], (it, ours[it], ref[it])
    assert np.max(np.abs(ours_eval["psnr"] - ref_eval["psnr"])) <= c["db"], (ours_eval["psnr"], ref_eval["psnr"])
