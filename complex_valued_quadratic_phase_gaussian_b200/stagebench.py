"""Run and time single stages of the fit iteration at a workload's size.

    python -m complex_valued_quadratic_phase_gaussian_b200.stagebench --stage blasm_fwd --workload rgb1080 --iters 3

Stages: ``blasm_fwd`` (rows, columns, inverse rows), ``blasm_adj`` (the three
adjoint passes), ``render`` (binning + splat forward of the drop-in path),
``splat_adj`` (the splat adjoint alone, on the lists of one forward call),
``loss`` (multi-plane loss + SSIM forward and dL/d(pred), with target noise),
``fit_step`` (whole fused fit iterations of the 1080p RGB fit, default FFT plan),
``mlp_train`` (training steps of the learned initialiser's MLP, 8192 tiles).
Only the buffers of that stage are allocated, so the process stays small
enough for kernel-level profiling. Prints one JSON line with the mean
milliseconds per call (CUDA events on the launching stream).
"""
import argparse
import json

import numpy as np
import torch

from .propagator import BlasmPlan, reference_distances, reference_pad_size

WORKLOADS = {
    "rgb1080": dict(W=1920, H=1080, C=3, N=96000, P=3, wl=[639e-9, 515e-9, 473e-9], pitch=3.74e-6, d_val=1e-3,
                    vd=1e-3),
    "gray256": dict(W=256, H=256, C=1, N=4096, P=3, wl=[515e-9], pitch=8e-6, d_val=1.5e-3, vd=1e-3),
    "gray4k": dict(W=3840, H=2160, C=1, N=200000, P=1, wl=[515e-9], pitch=3.74e-6, d_val=1e-3, vd=0.0),
}


def _field(C, H, W, seed=0):
    g = torch.Generator(device="cuda").manual_seed(seed)
    a = torch.rand((C, H, W), device="cuda", generator=g) * 1.2
    ph = torch.rand((C, H, W), device="cuda", generator=g) * 6.283
    return torch.polar(a, ph).contiguous()


def run(stage, workload, iters=3, warmup=1):
    w = WORKLOADS[workload]
    C, H, W, P = w["C"], w["H"], w["W"], w["P"]
    pad = reference_pad_size((W, H))
    dist = reference_distances(P, w["vd"], w["d_val"])
    times = []
    if stage in ("blasm_fwd", "blasm_adj"):
        plan = BlasmPlan(C, H, W, pad, w["wl"], dist, w["pitch"], aperture_radius=10 * max(W, H))
        f = _field(C, H, W)
        out = plan.forward(f)
        g = _field(P * C, H, W, seed=1).view(P, C, H, W) if stage == "blasm_adj" else None
        gin = torch.empty_like(f)
        for i in range(warmup + iters):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            if stage == "blasm_fwd":
                plan.forward(f, out=out)
            else:
                plan.backward(f, g, out=gin)
            e.record()
            torch.cuda.synchronize()
            if i >= warmup:
                times.append(s.elapsed_time(e))
    elif stage in ("render", "splat_adj"):
        from .rasterizer import render_backward, render_forward
        rng = np.random.default_rng(0)
        N = w["N"]
        means = torch.from_numpy(np.stack([rng.uniform(0, W, N), rng.uniform(0, H, N)], 1).astype(np.float32)).cuda()
        inv = torch.tensor([0.22, 0.01, 0.2], device="cuda").repeat(N, 1)
        col = torch.rand(N, C, device="cuda")
        ph = torch.rand(N, C, device="cuda") * 6.28
        z = torch.rand(N, device="cuda")
        radii = torch.full((N,), 12, dtype=torch.int32, device="cuda")
        k = (2 * np.pi / torch.tensor(w["wl"], dtype=torch.float32)).cuda()
        args = (means, inv, col, ph, z, z * 500, z + 4, k)
        _, pl, ranges = render_forward(*args, w["pitch"] ** 2, W, H, radii=radii)
        g = _field(C, H, W, seed=2)
        for i in range(warmup + iters):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            if stage == "render":
                render_forward(*args, w["pitch"] ** 2, W, H, radii=radii)
            else:
                render_backward(g, *args, pl, ranges, w["pitch"] ** 2, W, H)
            e.record()
            torch.cuda.synchronize()
            if i >= warmup:
                times.append(s.elapsed_time(e))
    elif stage == "loss":
        from .loss import MultiplaneLoss
        gen = torch.Generator(device="cuda").manual_seed(0)
        targets = torch.rand((P, C, H, W), device="cuda", generator=gen)
        pred = (0.9 * targets + 0.1 * torch.rand((P, C, H, W), device="cuda", generator=gen)).clamp_(0, 1)
        depth = torch.randint(0, P, (H, W), device="cuda", generator=gen, dtype=torch.int32).to(torch.uint8)
        lf = MultiplaneLoss(targets, depth, seed=1)
        out, grad = lf(pred, iteration=0)
        it = torch.zeros(1, dtype=torch.int32, device="cuda")
        for i in range(warmup + iters):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            lf(pred, iteration=it, out=out, grad_pred=grad)
            e.record()
            torch.cuda.synchronize()
            if i >= warmup:
                times.append(s.elapsed_time(e))
    elif stage == "fit_step":
        from .fit import FitConfig, Fitter, synthetic_init
        from .scenes import multiplane_targets_device, rgb_blobs
        img, depth = rgb_blobs(H, W, seed=0)
        targets, q = multiplane_targets_device(img, depth, P)
        cfg = FitConfig(img_size=(W, H), num_gaussians=w["N"], wavelengths=w["wl"], pixel_pitch=w["pitch"],
                        num_planes=P, d_val=w["d_val"], volume_depth=w["vd"], num_itrs=2000, seed=0)
        f = Fitter(cfg, targets, q, init=synthetic_init(cfg, 0))
        for i in range(warmup + iters):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            f.step()
            e.record()
            torch.cuda.synchronize()
            if i >= warmup:
                times.append(s.elapsed_time(e))
    elif stage == "mlp_train":
        from .mlp import TileMLP
        M = 8192
        g = torch.Generator(device="cuda").manual_seed(0)
        X = torch.rand((M, 1024), device="cuda", generator=g)
        T = torch.randn((M, 156), device="cuda", generator=g)
        wo = torch.ones(156, device="cuda")
        net = TileMLP(M)
        for i in range(warmup + iters):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            net.train_step(X, T, wo)
            e.record()
            torch.cuda.synchronize()
            if i >= warmup:
                times.append(s.elapsed_time(e))
    else:
        raise ValueError(stage)
    return {"stage": stage, "workload": workload, "ms": float(np.mean(times)), "iters": iters}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--stage", default="blasm_fwd", choices=["blasm_fwd", "blasm_adj", "render", "splat_adj", "loss", "fit_step", "mlp_train"])
    ap.add_argument("--workload", default="rgb1080", choices=sorted(WORKLOADS))
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    a = ap.parse_args()
    print(json.dumps(run(a.stage, a.workload, a.iters, a.warmup)))


if __name__ == "__main__":
    main()
