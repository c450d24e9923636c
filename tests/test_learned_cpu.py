"""CPU: host logic of the learned initialiser and the batched fitter's queue."""
import math

import numpy as np
import torch

from complex_valued_quadratic_phase_gaussian_b200 import learned as L
from complex_valued_quadratic_phase_gaussian_b200.batch import FitJob, shard


def test_tile_features_layout():
    H, W = 40, 50  # partial tiles on both axes
    img = torch.rand(3, H, W)
    depth = torch.rand(H, W)
    X = L.tile_features(img, depth, device="cpu")
    ty, tx = L.tile_grid(H, W)
    assert X.shape == (ty * tx, 1024)
    t = 1 * tx + 2  # tile row 1, column 2
    blk = X[t].view(4, 16, 16)
    assert torch.equal(blk[:3], img[:, 16:32, 32:48])
    assert torch.equal(blk[3], depth[16:32, 32:48])
    last = X[ty * tx - 1].view(4, 16, 16)  # the corner tile is zero beyond the image
    assert torch.all(last[:, H - 32:, :] == 0) and torch.all(last[:, :, W - 48:] == 0)


def test_encode_decode_round_trip():
    H, W = 48, 64
    cfg = L.scene_config(H, W, 10)
    raw = L.grid_init(cfg, seed=3)
    raw = {k: torch.as_tensor(v, dtype=torch.float32) for k, v in raw.items()}
    Y = L.encode(raw, H, W)
    assert Y.shape == (L.tile_grid(H, W)[0] * L.tile_grid(H, W)[1], 156)
    back = L.decode(Y, H, W)
    mu = lambda m: torch.stack([(torch.tanh(m[:, 0]) + 1) * W / 2, (torch.tanh(m[:, 1]) + 1) * H / 2], 1)
    assert torch.allclose(mu(back["means_2d"]), mu(raw["means_2d"]), atol=1e-3)
    for k in ("pre_act_scales", "colours", "pre_act_opacities", "curvature"):
        assert torch.allclose(back[k], raw[k].reshape(back[k].shape), atol=1e-6)
    assert torch.allclose(torch.remainder(back["pre_act_phase"], 2 * math.pi),
                          torch.remainder(raw["pre_act_phase"], 2 * math.pi), atol=1e-5)
    # every slot starts inside its own tile
    u = Y.view(-1, 12, 13)[..., :2]
    assert torch.all((u > 0) & (u < 1))


def test_shard_balances_cost_and_covers_every_job():
    cfgs = [L.scene_config(h, w, it) for h, w, it in
            [(256, 256, 500), (512, 512, 500), (128, 128, 200), (1080, 1920, 500), (768, 1024, 500), (64, 64, 100)]]
    jobs = [FitJob(c, None, None, c.num_itrs, tag=i) for i, c in enumerate(cfgs)]
    parts = [shard(jobs, r, 3) for r in range(3)]
    assert sorted(j.tag for p in parts for j in p) == list(range(len(jobs)))
    loads = [sum(j.cost() for j in p) for p in parts]
    assert max(loads) == cfgs[3].W * cfgs[3].H * 500  # the largest job alone bounds the makespan


def test_autotune_plans_factor_every_grid_of_the_configs():
    from complex_valued_quadratic_phase_gaussian_b200.autotune import candidates, plan_radices
    for n in (1152, 2816, 4480, 1664, 2176, 2688, 352, 480):
        for order in range(4):
            r = plan_radices(n, order)
            assert r is not None and int(np.prod(r)) == n
        assert len(set(tuple(plan_radices(n, o)) for o in range(4))) >= 2
    hs = candidates(2816, 4480)
    assert 11 in hs and len(hs) == len(set(hs))  # 11 = the default plan with its automatic register radix


def test_batched_fitter_pixel_budget_admission():
    """Host logic: a job is admitted while the resident fits' pixels stay within the budget;
    the first one always is."""
    from types import SimpleNamespace
    from complex_valued_quadratic_phase_gaussian_b200.batch import BatchedFitter
    job = lambda H, W: SimpleNamespace(cfg=SimpleNamespace(H=H, W=W), iters=10, cost=lambda: H * W * 10)
    bf = BatchedFitter.__new__(BatchedFitter)
    bf.pixel_budget, bf.active = 1000, []
    assert bf._fits_budget(job(100, 100))            # over the budget, but nothing is resident
    bf.active = [[job(20, 20), None, 5]]
    assert bf._fits_budget(job(20, 30))              # 400 + 600 = 1000
    assert not bf._fits_budget(job(20, 31))          # 400 + 620 > 1000
    bf.pixel_budget = None
    assert bf._fits_budget(job(1000, 1000))
