"""GPU: the batched fitter against single fits, and what the learned initialiser gains.

Batched fits run the same kernels as single fits (only the stream layout of the
graph differs), so their final per-plane PSNR matches a single fit of the same
job within 0.05 dB (the splat adjoint's float atomics make the bits differ).
The learned initialiser, trained as the bench trains it, must start above the
constant-init ablation and reach the plain (random-init) fit's final per-plane
PSNR on a held-out scene in at most half of the plain fit's time.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
START_MARGIN = 0.3  # dB, learned start PSNR over the constant-init ablation


@pytest.mark.parametrize("slots,budget", [(2, None), (8, 96 * 128 + 64 * 96)])
def test_batched_fitter_matches_single_fits(slots, budget):
    from complex_valued_quadratic_phase_gaussian_b200 import learned as L
    from complex_valued_quadratic_phase_gaussian_b200.batch import BatchedFitter, FitJob
    from complex_valued_quadratic_phase_gaussian_b200.fit import Fitter
    specs = [(48, 64, 30, 1), (64, 96, 50, 2), (96, 128, 40, 3), (32, 48, 20, 4)]
    jobs, scenes = [], {}
    for H, W, it, seed in specs:
        img, depth, targets, q = L.make_scene(H, W, seed)
        cfg = L.scene_config(H, W, it, seed=seed)
        scenes[seed] = (cfg, targets, q)
        jobs.append(FitJob(cfg, targets, q, it, init=L.grid_init(cfg, seed), tag=seed))
    bf = BatchedFitter(jobs, slots=slots, chunk=16, pixel_budget=budget)
    res = {r.tag: r for r in bf.run()}
    assert sorted(res) == [1, 2, 3, 4]
    for H, W, it, seed in specs:
        cfg, targets, q = scenes[seed]
        f = Fitter(L.scene_config(H, W, it, seed=seed), targets, q, init=L.grid_init(cfg, seed))
        f.run(it)
        ref = f.evaluate()["psnr"]
        assert res[seed].iters == it
        assert np.max(np.abs(res[seed].evaluation["psnr"] - ref)) < 0.05, (seed, res[seed].evaluation["psnr"], ref)
        assert not res[seed].overflowed


def test_learned_init_beats_constant_and_plain_init_on_a_held_out_scene():
    """What the network gains. Trained as bench.py trains it (two rounds of 64 batched fits of 256x256
    crops, 3000 MLP steps), on a held-out 512x512 scene the learned init must (a) start at least
    START_MARGIN dB (mean over the planes) above the ablation without the network (every slot at the
    mean training target), and (b) reach the plain fit's 500-iteration per-plane PSNR in at most half of
    the plain fit's time. At the bench's 1920x1080 scene the same training gives +0.8 to +1.2 dB at the
    start and 61-63 against 67-68 iterations to the goal; at 16 fits and 800 steps the network does not
    beat the ablation."""
    from complex_valued_quadratic_phase_gaussian_b200 import learned as L
    w, T2, info = L.train_initialiser(num_scenes=64, H=256, W=256, iters=400, steps=3000)
    assert info["pairs"] == 64 * 256
    res = L.time_to_psnr_experiment(w, T2, H=512, W=512, plain_iters=500, eval_every=50)
    print("learned-init experiment:", {k: res[k] for k in ("plain", "learned", "constant")})
    gain = float(np.mean(res["learned"]["psnr_start"]) - np.mean(res["constant"]["psnr_start"]))
    assert gain >= START_MARGIN, (gain, res)
    assert res["learned"]["fraction_of_plain"] is not None
    assert res["learned"]["fraction_of_plain"] <= 0.5, res
