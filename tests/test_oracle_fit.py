"""CPU: pin the float64 fit-iteration oracle to the reference fit loop (torch renderer, 3 iterations)."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import fit as ofit
from oracle import splat as osp

RAW = ("means_2d", "pre_act_scales", "pre_act_rotation", "colours", "pre_act_phase", "pre_act_opacities",
       "curvature")


def _lr_table(base, n, eta_min=1e-3):
    import torch
    p = torch.nn.Parameter(torch.zeros(1))
    opt = torch.optim.SGD([p], lr=base)
    sch = torch.optim.lr_scheduler.CosineAnnealingLR(opt, T_max=n, eta_min=eta_min)
    out = []
    for _ in range(n):
        out.append(opt.param_groups[0]["lr"])
        opt.step()
        sch.step()
    return out


@pytest.mark.parametrize("name", ["fit_rgb", "fit_gray"])
def test_oracle_fit_iterations_match_reference_loop(golden, name):
    g = golden(name)
    W, H = int(g["W"]), int(g["H"])
    lrs = [0.01, 0.005, 0.0025, 0.025, 0.001, 0.001]
    orc = ofit.FitOracle({k: g["init_" + k] for k in RAW}, W, H, list(g["wavelengths"]), float(g["pitch"]),
                         list(g["pad"]), list(g["distances"]), float(g["aperture"]), lrs,
                         means_lr_table=_lr_table(0.01, int(g["num_itrs"])), cull=osp.CULL_TORCH64_3SIGMA,
                         warmup_iters=int(g["warmup"]), seed=int(g["seed"]))
    for it in range(int(g["iters"])):
        o = orc.step(g["targets"], g["depth_plane"], inject_noise=True)
        assert abs(o["loss"] - g["loss"][it]) < 1e-6 * g["loss"][it]
        for k in RAW:
            ref = g[f"it{it}_{k}"].astype(np.float64)
            assert rel_l2(orc.raw[k], ref) < 1e-5, (it, k)
            orc.raw[k] = ref.copy()  # re-sync (the reference runs in float32)
