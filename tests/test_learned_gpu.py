"""GPU: the batched fitter against single fits, and what the learned initialiser gains.

Batched fits run the same kernels as single fits (only the stream layout of the
graph differs), so their final per-plane PSNR matches a single fit of the same
job within 0.05 dB (the splat adjoint's float atomics make the bits differ).
The learned initialiser, trained here on 16 small fits, must reach the plain
(random-init) fit's final per-plane PSNR on a held-out scene in at most half of
the plain fit's time.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


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


def test_learned_init_beats_plain_init_on_a_held_out_scene():
    from complex_valued_quadratic_phase_gaussian_b200 import learned as L
    w, T2, info = L.train_initialiser(num_scenes=16, H=128, W=128, iters=200, steps=800)
    assert info["pairs"] == 16 * 64
    res = L.time_to_psnr_experiment(w, T2, H=256, W=256, plain_iters=300, eval_every=25)
    print("learned-init experiment:", {k: res[k] for k in ("plain", "learned", "constant")})
    assert res["learned"]["fraction_of_plain"] is not None
    assert res["learned"]["fraction_of_plain"] <= 0.5, res
