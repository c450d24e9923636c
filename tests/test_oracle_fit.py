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


@pytest.mark.parametrize("name", ["fit_rgb", "fit_gray"])
def test_timed_torch_port_matches_reference_loop(golden, name):
    """The torch port that bench.py times as the reference implementation (oracle/torch_port.py)
    runs the same iterations as the reference loop itself: loss within 1e-5 relative and
    parameters within 1e-5 relative L2 per iteration, on the reference-loop goldens."""
    import torch
    from oracle import loss as oloss
    from oracle.torch_port import ReferencePipeline
    g = golden(name)
    W, H, C, P = int(g["W"]), int(g["H"]), int(g["C"]), int(g["P"])
    seed = int(g["seed"])
    pipe = ReferencePipeline({k: g["init_" + k] for k in RAW}, (W, H), list(g["wavelengths"]), float(g["pitch"]),
                             list(g["pad"]), list(g["distances"]), float(g["aperture"]), g["targets"],
                             g["depth_plane"], renderer="torch", warmup_iters=int(g["warmup"]),
                             num_itrs=int(g["num_itrs"]), device="cpu",
                             noise=lambda it: oloss.plane_noise((P, C, H, W), seed, it))
    for it in range(int(g["iters"])):
        pipe.step()
        assert abs(pipe.last_loss - g["loss"][it]) < 1e-5 * g["loss"][it], (it, pipe.last_loss, g["loss"][it])
        for k in RAW:
            got = pipe.params[k].detach().numpy().astype(np.float64)
            ref = g[f"it{it}_{k}"].astype(np.float64)
            assert rel_l2(got, ref) < 1e-5, (it, k, rel_l2(got, ref))
            with torch.no_grad():  # re-sync, as the reference runs in float32
                pipe.params[k].copy_(torch.from_numpy(g[f"it{it}_{k}"]))
