"""Float64 finite differences of the fit loss, one Gaussian at a time. TEST INFRASTRUCTURE ONLY.

The checker of the fused gradient against central finite differences. The loss is
the oracle's noise-free fit loss (oracle/fit.py: preprocess -> culled splat ->
soft_window_pad + amplitude clamp -> BLASM to every plane -> multi-plane loss +
SSIM), restated here in torch float64 so that the ~1,000 loss evaluations of a
64-primitive x 9-parameter check can run on any torch device:

* the splat field is incremental: the base field U0 is the numpy oracle's
  (oracle/splat.py, the cull rule's lists at the base parameters), and a
  perturbed Gaussian g changes U0 only on the pixels of g's base tile lists
  (the lists are held fixed, as they are for an infinitesimal change), by
  u_g(perturbed) - u_g(base) with u_g the reference's per-pixel term
  (cuda/forward.cu:131-151, model_2d_gaussian_rgb.py:351-370);
* the chain restates oracle/blasm.py:chain_forward (model_2d_gaussian_rgb.py:186-241,
  train_2d_gaussian_rgb.py:89-95, utils/propagator.py:41-64, 248-290) with the
  same transfer multipliers (oracle.blasm.multiplier). The reference builds the
  replicate guard band of soft_window_pad under no_grad (model_2d_gaussian_rgb.py:
  207-226), so its gradient, and the fused one, treat the band as a constant: the
  differences here keep the band at its base value (from U0) and move only the
  image part;
* the loss restates oracle/loss.py:multiplane_loss (utils/propagator.py:417-449,
  utils/data_utils.py:22-41) without noise, with the oracle's SSIM (oracle/ssim.py).

tests/test_oracle_fd64.py pins it to the numpy oracle.
"""
import numpy as np
import torch

from . import blasm as ob
from . import preprocess as opre
from . import splat as osp
from . import ssim as ossim

RAW_KEYS = opre.RAW_KEYS


class FiniteDifferenceLoss:
    def __init__(self, raw, W, H, wavelengths, pixel_pitch, pad, distances, aperture_radius, targets, depth_plane,
                 curv_mode="scale_aware", cull=osp.CULL_CUDA16_5SIGMA, device="cpu", eta=0.9,
                 weights=(1.0, 1.0, 1.0), ssim_weight=0.005):
        self.raw = {k: np.asarray(v, dtype=np.float64).copy() for k, v in raw.items()}
        self.W, self.H = W, H
        self.wl, self.dx, self.pad = list(wavelengths), float(pixel_pitch), list(pad)
        self.dist = list(distances)
        self.curv_mode, self.cull, self.eta = curv_mode, cull, eta
        self.weights, self.ssim_w = weights, ssim_weight
        self.dev = torch.device(device)
        self.C = self.raw["colours"].shape[1]
        self.k = (np.float32(2 * np.pi) / np.asarray(self.wl, dtype=np.float32)).astype(np.float64)
        self.dxy2 = float(np.float32(self.dx * self.dx))
        act = self._activate(self.raw)
        self.act = act
        pl, ranges = osp.bin_lists(act["means"].astype(np.float32), W, H, cull, radii=act["radii"],
                                   radius3=act["radius3"].astype(np.float32))
        self.pl, self.ranges = pl, ranges
        U0 = osp.splat_forward(act["means"], act["inv_cov"], act["colours"], act["phase"], act["opac"], act["curv"],
                               act["area"], self.k, self.dxy2, W, H, cull=cull, point_list=pl, ranges=ranges)
        self.U0 = torch.from_numpy(U0).to(self.dev)
        # pixels of each Gaussian's base lists (tile rows/cols of the cull rule)
        _, self.lgx, self.lgy = osp.list_grid(cull, W, H)
        pH, pW = self.pad
        NH, NW = 2 * pH, 2 * pW
        self.M = torch.stack([torch.stack([torch.from_numpy(ob.multiplier(NH, NW, self.dx, self.wl[c], float(z),
                                                                          aperture_radius))
                                           for c in range(self.C)]) for z in self.dist]).to(self.dev)
        ph, pw = (pH - H) // 2, (pW - W) // 2
        self.rows = torch.from_numpy(np.clip(np.arange(pH) - ph, 0, H - 1)).to(self.dev)
        self.cols = torch.from_numpy(np.clip(np.arange(pW) - pw, 0, W - 1)).to(self.dev)
        self.win = torch.from_numpy(np.outer(ob.taper_1d(pH, ph, H), ob.taper_1d(pW, pw, W))).to(self.dev)
        self.T = torch.as_tensor(np.asarray(targets, dtype=np.float64), device=self.dev)
        q = np.asarray(depth_plane)
        self.masks = torch.stack([torch.from_numpy((q == p).astype(np.float64)) for p in range(len(self.dist))]).to(
            self.dev)

    def _activate(self, raw):
        return opre.activate(raw, self.W, self.H, self.wl, self.dx, curv_mode=self.curv_mode, eta=self.eta)

    # -- loss of a field -------------------------------------------------------------------
    def loss_of_field(self, U, band=None):
        """Noise-free loss of a splat field U [C,H,W] (complex128 tensor); the replicate guard
        band comes from `band` (default U itself)."""
        pH, pW = self.pad
        NH, NW = 2 * pH, 2 * pW
        x = (U if band is None else band)[:, self.rows][:, :, self.cols]
        ph, pw = (pH - self.H) // 2, (pW - self.W) // 2
        if band is not None:
            x = x.clone()
            x[:, ph:ph + self.H, pw:pw + self.W] = U
        x = x * self.win
        a = torch.abs(x)
        x = torch.where(a > 1.0, x / torch.where(a > 0, a, torch.ones_like(a)), x)
        E = torch.zeros((self.C, NH, NW), dtype=torch.complex128, device=self.dev)
        r0, c0 = NH // 2 - pH // 2, NW // 2 - pW // 2
        E[:, r0:r0 + pH, c0:c0 + pW] = x
        F = torch.fft.fft2(E)
        H, W = self.H, self.W
        o0, o1 = NH // 2 - H // 2, NW // 2 - W // 2
        n = self.C * H * W
        w0, w1, w2 = self.weights
        total = torch.zeros((), dtype=torch.float64, device=self.dev)
        for p in range(len(self.dist)):
            V = torch.fft.ifft2(self.M[p] * F)[:, o0:o0 + H, o1:o1 + W]
            pred = torch.clamp(V.real ** 2 + V.imag ** 2, 0.0, 1.0)
            t = self.T[p]
            m = self.masks[p][None]
            d0, d1, d2 = pred - t, pred * m - t * m, pred * t - t * t
            total = total + (w0 * (d0 ** 2).sum() + w1 * (d1 ** 2).sum() + w2 * (d2 ** 2).sum()) / n
            s = ossim.ssim_torch(pred[None], t[None]).mean()
            total = total + self.ssim_w * (1.0 - s)
        return float(total)

    def base_loss(self):
        return self.loss_of_field(self.U0)

    # -- one Gaussian's term -----------------------------------------------------------------
    def _pixels(self, g):
        tiles = osp._tiles_of(g, self.cull, self.act["means"].astype(np.float32), self.W, self.H, self.act["radii"],
                              self.act["radius3"].astype(np.float32), self.lgx, self.lgy)
        ys, xs = [], []
        edge = 16 if self.cull == osp.CULL_CUDA16_5SIGMA else 64
        for t in tiles:
            tx, ty = t % self.lgx, t // self.lgx
            y0, x0 = ty * edge, tx * edge
            yy, xx = np.meshgrid(np.arange(y0, min(y0 + edge, self.H)), np.arange(x0, min(x0 + edge, self.W)),
                                 indexing="ij")
            ys.append(yy.ravel())
            xs.append(xx.ravel())
        if not ys:
            return np.zeros(0, np.int64), np.zeros(0, np.int64)
        return np.concatenate(ys), np.concatenate(xs)

    def _term(self, act, j, ys, xs):
        dx = act["means"][j, 0] - xs.astype(np.float64)
        dy = act["means"][j, 1] - ys.astype(np.float64)
        i00, i01, i11 = act["inv_cov"][j]
        mahal = dx * (i00 * dx + i01 * dy) + dy * (i01 * dx + i11 * dy)
        alpha = act["opac"][j] * np.exp(np.maximum(-0.5 * mahal, -50.0))
        base = 0.5 * act["curv"][j] * mahal * act["area"][j] * self.dxy2
        return np.stack([act["colours"][j, c] * alpha * np.exp(1j * (act["phase"][j, c] + self.k[c] * base))
                         for c in range(self.C)])

    def loss_with(self, g, key, index, value):
        """Loss with raw parameter `key`[g, index] (index None for a 1-D tensor) set to `value`."""
        ys, xs = self._pixels(g)
        one = {k: v[g:g + 1].copy() for k, v in self.raw.items()}
        if index is None:
            one[key][0] = value
        else:
            one[key][0, index] = value
        new = self._activate(one)
        d = self._term(new, 0, ys, xs) - self._term(self.act, g, ys, xs)
        U = self.U0.clone()
        if ys.size:
            yt = torch.from_numpy(ys).to(self.dev)
            xt = torch.from_numpy(xs).to(self.dev)
            U[:, yt, xt] += torch.from_numpy(d).to(self.dev)
        return self.loss_of_field(U, band=self.U0)

    def central_difference(self, g, key, index=None, h=1e-3):
        v = self.raw[key][g] if index is None else self.raw[key][g, index]
        return (self.loss_with(g, key, index, v + h) - self.loss_with(g, key, index, v - h)) / (2.0 * h)
