"""Oracle: one full fit iteration in float64 numpy. Test infrastructure only.

Chains the restatements of the reference loop body (train_2d_gaussian_rgb.py:187-211):
preprocess (oracle.preprocess) -> binning + splat (oracle.splat) -> pad, clamp and
BLASM (oracle.blasm) -> multi-plane loss + SSIM (oracle.loss) -> adjoints ->
nan_to_num -> clip_grad_norm_(1.0) -> Adan (oracle.adan), with the means cosine
schedule (train_2d_gaussian_rgb.py:58-70) and the curvature warm-up (:147-185).
"""
import numpy as np

from . import adan as oadan
from . import blasm as ob
from . import loss as ol
from . import preprocess as opre
from . import splat as osp

GROUPS = [("means", ["means_2d"]), ("scales", ["pre_act_scales"]), ("amplitude_phase", ["colours", "pre_act_phase"]),
          ("opacity", ["pre_act_opacities"]), ("rotation", ["pre_act_rotation"]), ("curvature", ["curvature"])]


class FitOracle:
    def __init__(self, raw, W, H, wavelengths, pixel_pitch, pad, distances, aperture_radius, lrs, means_lr_table=None,
                 cull=osp.CULL_CUDA16_5SIGMA, curv_mode="scale_aware", curv_trainable=True, warmup_iters=0,
                 eta=0.9, max_grad_norm=1.0, weights=(1.0, 1.0, 1.0), ssim_weight=0.005, noise_ratio=1e-3,
                 seed=0):
        self.raw = {k: np.asarray(v, dtype=np.float64).copy() for k, v in raw.items()}
        self.W, self.H = W, H
        self.wl, self.dx, self.pad = list(wavelengths), pixel_pitch, pad
        self.dist, self.ap = list(distances), aperture_radius
        self.cull, self.curv_mode = cull, curv_mode
        self.curv_trainable, self.warmup = curv_trainable, warmup_iters
        self.eta, self.max_norm = eta, max_grad_norm
        self.weights, self.ssim_w, self.noise_ratio, self.seed = weights, ssim_weight, noise_ratio, seed
        self.lr_table = means_lr_table
        self.opt = oadan.Adan([{"params": names, "lr": lr} for (_, names), lr in zip(GROUPS, lrs)])
        self.it = 0

    def forward(self, targets, depth_plane, noise=None):
        C = self.raw["colours"].shape[1]
        act = opre.activate(self.raw, self.W, self.H, self.wl, self.dx, curv_mode=self.curv_mode, eta=self.eta)
        k = (np.float32(2 * np.pi) / np.asarray(self.wl, dtype=np.float32)).astype(np.float64)
        dxy2 = float(np.float32(self.dx * self.dx))
        if self.cull == osp.CULL_NONE:
            pl, ranges = None, None
        else:
            pl, ranges = osp.bin_lists(act["means"].astype(np.float32), self.W, self.H, self.cull,
                                       radii=act["radii"], radius3=act["radius3"].astype(np.float32))
        args = (act["means"], act["inv_cov"], act["colours"], act["phase"], act["opac"], act["curv"], act["area"], k,
                dxy2, self.W, self.H)
        U = osp.splat_forward(*args, cull=self.cull, point_list=pl, ranges=ranges)
        V = ob.chain_forward(U, self.pad[0], self.pad[1], self.wl, self.dist, self.dx, aperture_radius=self.ap)
        loss, mse, ssim, gV = ol.multiplane_loss(V, targets, depth_plane, self.weights, self.ssim_w, noise,
                                                 self.noise_ratio)
        return dict(act=act, args=args, pl=pl, ranges=ranges, U=U, V=V, loss=loss, mse=mse, ssim=ssim, gV=gV)

    def step(self, targets, depth_plane, inject_noise=True):
        P = len(self.dist)
        C = self.raw["colours"].shape[1]
        noise = ol.plane_noise((P, C, self.H, self.W), self.seed, self.it) if inject_noise else None
        f = self.forward(targets, depth_plane, noise)
        gU = ob.chain_backward(f["U"], f["gV"], self.pad[0], self.pad[1], self.wl, self.dist, self.dx,
                               aperture_radius=self.ap)
        gs = osp.splat_backward(gU, *f["args"], cull=self.cull, point_list=f["pl"], ranges=f["ranges"])
        grads = opre.activate_backward(f["act"], *gs[:2], gs[2], gs[3], gs[4], gs[5], gs[6])
        grads = {k: np.nan_to_num(v, nan=0.0, posinf=0.0, neginf=0.0) for k, v in grads.items()}
        curv_active = self.curv_trainable and self.it >= self.warmup
        if not curv_active:
            grads["curvature"] = None
        names = list(opre.RAW_KEYS)
        clipped, norm = oadan.clip_grad_norm([grads[n] for n in names], self.max_norm)
        grads = dict(zip(names, clipped))
        if self.lr_table is not None:
            self.opt.groups[0]["lr"] = self.lr_table[min(self.it, len(self.lr_table) - 1)]
        self.opt.step(self.raw, grads)
        self.it += 1
        return dict(loss=f["loss"], mse=f["mse"], ssim=f["ssim"], norm=norm, grads=grads, V=f["V"], U=f["U"])
