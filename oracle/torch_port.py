"""Torch port of the reference fit loop -- the timed baseline (TEST/BENCH INFRASTRUCTURE ONLY).

A restatement, in the reference's own torch operation order, of one iteration of
the reference fit loop (train_2d_gaussian_rgb.py:187-211):

* renderer 'torch': the 64-px tile loop with 3-sigma culling and batches of 1024
  Gaussians (model_2d_gaussian_rgb.py:269-422), run on any device;
* renderer 'cuda': the reference's own compiled CUDA rasterizer (oracle/_ref,
  built from the reference sources by oracle/build_ref.py) behind a
  QPFRender-style autograd wrapper (cuda/rasterizer.py:36-59) with the
  reference's culling radius (model_2d_gaussian_rgb.py:424-439);
* soft_window_pad (model_2d_gaussian_rgb.py:186-241);
* reconstruct() and the propagator (train_2d_gaussian_rgb.py:89-95,
  utils/propagator.py:248-290) with torch.fft, one (frame, plane, channel) at a
  time with the cached transfer functions (oracle/odak_restated.py);
* multiplane loss with noise + SSIM per plane, the per-iteration PSNR of plane 0
  copied to the host and loss.item() (train_2d_gaussian_rgb.py:191-202);
* nan_to_num, clip_grad_norm_(1.0), Adan (foreach=False), the means cosine schedule.

It is what bench.py times as the reference CPU implementation (on the host cores)
and as the reference GPU pipeline; it is never part of the product.
"""
import glob
import importlib.util
import math
import os

import numpy as np
import torch
import torch.nn.functional as F

from . import odak_restated as odr
from . import ssim as ossim

RAW_KEYS = ("means_2d", "pre_act_scales", "pre_act_rotation", "colours", "pre_act_phase", "pre_act_opacities",
            "curvature")


def load_reference_extension():
    """Import the reference qpf_2d_cuda extension built into oracle/_ref/ (None if absent)."""
    here = os.path.dirname(os.path.abspath(__file__))
    so = sorted(glob.glob(os.path.join(here, "_ref", "qpf_2d_cuda*.so")))
    if not so:
        return None
    spec = importlib.util.spec_from_file_location("qpf_2d_cuda", so[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _RefQPFRender(torch.autograd.Function):
    """QPFRender of cuda/rasterizer.py:36-59 over the reference's compiled extension."""

    @staticmethod
    def forward(ctx, ext, means_2d, inv_cov, colours, phase, opacities, curvature, area, radii, k, dxy2, W, H):
        C = colours.shape[1]
        args = [t.contiguous() for t in (means_2d, inv_cov, colours, phase, opacities, curvature, area)]
        out_r, out_i, point_list, ranges = ext.qpf_render_forward(*args, radii.contiguous().int(), k.contiguous(),
                                                                  float(dxy2), int(W), int(H), int(C))
        ctx.save_for_backward(*args, k.contiguous(), point_list, ranges)
        ctx.cfg = (ext, float(dxy2), int(W), int(H), int(C))
        return torch.complex(out_r, out_i)

    @staticmethod
    def backward(ctx, grad_out):
        means, inv_cov, colours, phase, opac, curv, area, k, point_list, ranges = ctx.saved_tensors
        ext, dxy2, W, H, C = ctx.cfg
        d = ext.qpf_render_backward(grad_out.real.contiguous(), grad_out.imag.contiguous(), means, inv_cov, colours,
                                    phase, opac, curv, area, k, point_list, ranges, dxy2, W, H, C)
        return (None, d[0], d[1], d[2], d[3], d[4], d[5], d[6], None, None, None, None, None)


def soft_window_pad(h, pad):
    C, H, W = h.shape
    pH, pW = pad
    ph, pw = (pH - H) // 2, (pW - W) // 2
    phb, pwr = pH - H - ph, pW - W - pw
    with torch.no_grad():
        rep = torch.complex(F.pad(h.real.unsqueeze(0), (pw, pwr, ph, phb), mode="replicate").squeeze(0),
                            F.pad(h.imag.unsqueeze(0), (pw, pwr, ph, phb), mode="replicate").squeeze(0))
    zero = torch.complex(F.pad(h.real.unsqueeze(0), (pw, pwr, ph, phb)).squeeze(0),
                         F.pad(h.imag.unsqueeze(0), (pw, pwr, ph, phb)).squeeze(0))
    mask = torch.zeros(1, pH, pW, device=h.device)
    mask[:, ph:ph + H, pw:pw + W] = 1.0

    def taper(total, start, size):
        w = torch.zeros(total, device=h.device)
        w[start:start + size] = 1.0
        if start > 0:
            t = torch.arange(start, device=h.device, dtype=torch.float32)
            w[:start] = 0.5 * (1.0 - torch.cos(torch.pi * (t + 1.0) / start))
        r = start + size
        n = total - r
        if n > 0:
            t = torch.arange(n, device=h.device, dtype=torch.float32)
            w[r:] = 0.5 * (1.0 + torch.cos(torch.pi * (t + 1.0) / n))
        return w

    win = torch.outer(taper(pH, ph, H), taper(pW, pw, W)).unsqueeze(0)
    return (zero + rep * (1.0 - mask)) * win


class ReferencePipeline:
    """One reference fit iteration per step(), on `device`, with renderer 'torch' or 'cuda'."""

    def __init__(self, raw, img_size, wavelengths, pixel_pitch, pad, distances, aperture, targets, depth_plane,
                 renderer="torch", lrs=(0.01, 0.005, 0.0025, 0.025, 0.001, 0.001), warmup_iters=400, num_itrs=2001,
                 device="cpu", ext=None, curv_nyquist=0.9, noise=None):
        """noise: None draws the target noise with torch.randn_like as the reference loop does
        (utils/propagator.py:432); a callable noise(iteration) -> [P, C, H, W] standard normals
        injects given noise instead (the parity tests use the oracle's counter-based normals)."""
        self.dev = torch.device(device)
        self.W, self.H = img_size
        self.wl = list(wavelengths)
        self.C = len(self.wl)
        self.dx = pixel_pitch
        self.pad = list(pad)
        self.dist = list(distances)
        self.renderer = renderer
        self.ext = ext
        self.eta = curv_nyquist
        self.params = {k: torch.nn.Parameter(torch.as_tensor(raw[k], dtype=torch.float32).to(self.dev).clone())
                       for k in RAW_KEYS}
        self.targets = torch.as_tensor(targets, dtype=torch.float32, device=self.dev)
        q = torch.as_tensor(depth_plane, device=self.dev)
        self.masks = torch.stack([(q == p).float().unsqueeze(0).expand(self.C, -1, -1) for p in range(len(self.dist))])
        self.wl_t = torch.tensor(self.wl, dtype=torch.float32, device=self.dev)
        pH, pW = self.pad
        x = torch.linspace(-pH, pH, 2 * pH)
        y = torch.linspace(-pW, pW, 2 * pW)
        X, Y = torch.meshgrid(x, y, indexing="ij")
        self.aperture = (torch.sqrt(X ** 2 + Y ** 2) < aperture).float().to(self.dev)
        self.kernels = {}
        groups = [("means_2d",), ("pre_act_scales",), ("colours", "pre_act_phase"), ("pre_act_opacities",),
                  ("pre_act_rotation",), ("curvature",)]
        self.groups = [{"params": list(g), "lr": lr, "step": 0} for g, lr in zip(groups, lrs)]
        self.state = {}
        self.warmup = warmup_iters
        p = torch.nn.Parameter(torch.zeros(1))
        self._sgd = torch.optim.SGD([p], lr=lrs[0])
        self._sched = torch.optim.lr_scheduler.CosineAnnealingLR(self._sgd, T_max=max(1, num_itrs), eta_min=1e-3)
        self.it = 0
        self.noise = noise
        self._noise_now = None

    # -- render ---------------------------------------------------------------------------
    def activations(self):
        P_ = self.params
        mt = torch.tanh(P_["means_2d"])
        means = torch.zeros_like(mt)
        means[:, 0] = (mt[:, 0] + 1) * 0.5 * self.W
        means[:, 1] = (mt[:, 1] + 1) * 0.5 * self.H
        scales = torch.exp(P_["pre_act_scales"]) + 0.1
        rot = P_["pre_act_rotation"]
        phase = P_["pre_act_phase"] % (2.0 * np.pi)
        opac = torch.sigmoid(P_["pre_act_opacities"])
        lam = float(min(self.wl)) if self.C == 3 else float(self.wl[0])
        sigma = scales.max(dim=1).values
        cmax = self.eta * lam / (6.0 * sigma * (self.dx ** 2) + 1e-20)
        curv = cmax * torch.tanh(P_["curvature"])
        c, s = torch.cos(rot), torch.sin(rot)
        sx, sy = scales[:, 0], scales[:, 1]
        c00 = sx * sx * c * c + sy * sy * s * s + 0.1
        c01 = (sx * sx - sy * sy) * c * s
        c11 = sx * sx * s * s + sy * sy * c * c + 0.1
        det = (c00 * c11 - c01 * c01).clamp(min=1e-10)
        inv = (c11 / det, -c01 / det, c00 / det)
        return means, scales, phase, opac, curv, (c00, c01, c11), inv

    def render(self, tile_rows=None):
        means, scales, phase, opac, curv, cov, inv = self.activations()
        colours = self.params["colours"]
        k = 2 * np.pi / self.wl_t
        dxy2 = self.dx ** 2
        C, H, W = self.C, self.H, self.W
        c00, c01, c11 = cov
        if self.renderer == "cuda":
            inv_cov = torch.stack(inv, -1)
            area = (scales[:, 0] * scales[:, 1]).abs()
            with torch.no_grad():
                mid = 0.5 * (c00 + c11)
                disc = torch.sqrt(((c00 - c11) * 0.5) ** 2 + c01 ** 2)
                radii = (5.0 * torch.sqrt(mid + disc)).ceil().to(torch.int32)
            return _RefQPFRender.apply(self.ext, means, inv_cov, colours, phase, opac, curv, area, radii, k.contiguous(),
                                       dxy2, W, H)
        holo = torch.zeros((C, H, W), dtype=torch.complex64, device=self.dev)
        cf = (colours * torch.exp(1j * phase)).to(torch.complex64)
        mid = 0.5 * (c00 + c11)
        disc = torch.sqrt(((c00 - c11) * 0.5) ** 2 + c01 ** 2)
        radius = 3.0 * torch.sqrt(mid + disc)
        tdh = math.sqrt(32.0 ** 2 + 32.0 ** 2)
        ys = list(range(0, H, 64))
        if tile_rows is not None:
            ys = ys[tile_rows[0]:tile_rows[1]]
        for y0 in ys:
            y1 = min(y0 + 64, H)
            for x0 in range(0, W, 64):
                x1 = min(x0 + 64, W)
                cx, cy = (x0 + x1) / 2.0, (y0 + y1) / 2.0
                mask = (means[:, 0] - cx) ** 2 + (means[:, 1] - cy) ** 2 < (radius + tdh) ** 2
                xs_ = torch.arange(x0, x1, device=self.dev, dtype=torch.float32)
                ys_ = torch.arange(y0, y1, device=self.dev, dtype=torch.float32)
                gy, gx = torch.meshgrid(ys_, xs_, indexing="ij")
                pts = torch.stack([gx, gy], -1).reshape(1, -1, 2)
                acc = torch.zeros((C, pts.shape[1]), dtype=torch.complex64, device=self.dev)
                if bool(mask.any()):
                    mm, i0, i1, i2 = means[mask], inv[0][mask], inv[1][mask], inv[2][mask]
                    mo, mc, mcv, ms = opac[mask].unsqueeze(1), cf[mask], curv[mask].unsqueeze(1), scales[mask]
                    for b0 in range(0, mm.shape[0], 1024):
                        b1 = b0 + 1024
                        d = pts - mm[b0:b1].unsqueeze(1)
                        dx_, dy_ = d[..., 0], d[..., 1]
                        mah = dx_ * dx_ * i0[b0:b1, None] + 2 * dx_ * dy_ * i1[b0:b1, None] + dy_ * dy_ * i2[b0:b1, None]
                        G = torch.exp(torch.clamp(-0.5 * mah, min=-50))
                        al = mo[b0:b1] * G
                        ar = (ms[b0:b1, 0] * ms[b0:b1, 1]).abs().unsqueeze(1)
                        base = 0.5 * mcv[b0:b1] * mah * ar * dxy2
                        mod = torch.polar(al.unsqueeze(0).expand(C, -1, -1), k.view(C, 1, 1) * base.unsqueeze(0))
                        acc = acc + torch.einsum("cbp, bc -> cp", mod, mc[b0:b1])
                holo[:, y0:y1, x0:x1] += acc.view(C, y1 - y0, x1 - x0)
        return holo

    # -- propagate ------------------------------------------------------------------------
    def transfer(self, p, c):
        key = (p, c)
        if key not in self.kernels:
            pH, pW = self.pad
            H = odr.get_propagation_kernel(2 * pH, 2 * pW, self.dx, self.wl[c], self.dist[p])
            self.kernels[key] = H.to(self.dev)
        return self.kernels[key]

    def propagate(self, U, planes=None, channels=None):
        """reconstruct(): intensities [P, C, H, W] (cropped to the image) as in train_2d_gaussian_rgb.py:89-95, 193."""
        pH, pW = self.pad
        phase = torch.angle(U) % (2 * math.pi)
        amp = torch.clamp(torch.abs(U), min=0.0, max=1.0)
        planes = range(len(self.dist)) if planes is None else planes
        channels = range(self.C) if channels is None else channels
        out = []
        for p in planes:
            row = []
            for c in channels:
                f = amp[c] * torch.cos(phase[c]) + 1j * amp[c] * torch.sin(phase[c])
                f = odr.zero_pad(f)
                A = self.aperture
                Hk = self.transfer(p, c) * A
                U1 = torch.fft.fftshift(torch.fft.fft2(f)) * A
                r = torch.fft.ifft2(torch.fft.ifftshift(Hk * U1))
                r = odr.crop_center(r)
                I = torch.abs(r) ** 2
                row.append(odr.crop_center(I, size=(self.H, self.W)))
            out.append(torch.stack(row))
        return torch.stack(out)

    # -- loss -----------------------------------------------------------------------------
    def loss(self, I, planes=None, host_metrics=True):
        total = 0.0
        planes = range(I.shape[0]) if planes is None else planes
        for i, p in enumerate(planes):
            pred = torch.clamp(I[i], 0.0, 1.0)
            t = self.targets[p]
            m = self.masks[p]
            l2 = F.mse_loss(pred, t)
            z = torch.randn_like(t) if self._noise_now is None else self._noise_now[p]
            nt = t + z * 1e-3 * (t.max() - t.min())
            total = total + l2 + F.mse_loss(pred * m, nt * m) + F.mse_loss(pred * nt, nt * nt)
            s = ossim.ssim_torch(pred.unsqueeze(0), t.unsqueeze(0)).mean()
            total = total + 0.025 * 0.2 * (1 - s)
            if host_metrics and p == 0:
                a, b = pred.detach().cpu().numpy(), t.detach().cpu().numpy()
                self.last_psnr = 10 * np.log10(1.0 / max(float(np.mean((a - b) ** 2)), 1e-30))
        return total

    # -- optimiser ------------------------------------------------------------------------
    @torch.no_grad()
    def adan_step(self, trainable):
        b1, b2, b3 = 0.98, 0.92, 0.99
        for g in self.groups:
            g["step"] += 1
            st_ = g["step"]
            bc1, bc2, bc3 = 1 - b1 ** st_, 1 - b2 ** st_, 1 - b3 ** st_
            for name in g["params"]:
                p = self.params[name]
                if name not in trainable or p.grad is None:
                    continue
                grad = p.grad
                s = self.state.setdefault(name, {})
                if not s:
                    s["m"], s["v"], s["d"] = torch.zeros_like(p), torch.zeros_like(p), torch.zeros_like(p)
                if "ng" not in s or st_ == 1:
                    s["ng"] = grad.clone().mul_(-1.0)
                ng = s["ng"].add_(grad)
                s["m"].mul_(b1).add_(grad, alpha=1 - b1)
                s["d"].mul_(b2).add_(ng, alpha=1 - b2)
                ng.mul_(b2).add_(grad)
                s["v"].mul_(b3).addcmul_(ng, ng, value=1 - b3)
                denom = (s["v"].sqrt() / math.sqrt(bc3)).add_(1e-8)
                p.addcdiv_(s["m"], denom, value=-g["lr"] / bc1)
                p.addcdiv_(s["d"], denom, value=-g["lr"] * b2 / bc2)
                ng.zero_().add_(grad, alpha=-1.0)

    def gradients(self, sanitize=True):
        """The raw-parameter gradients of one iteration's loss after nan_to_num (or before it, with
        sanitize=False), before the clip and the update (train_2d_gaussian_rgb.py:187-208);
        nothing is changed."""
        trainable = set(RAW_KEYS) if self.it >= self.warmup else set(RAW_KEYS) - {"curvature"}
        for k, p in self.params.items():
            p.grad = None
            p.requires_grad_(k in trainable)
        U = soft_window_pad(self.render(), self.pad)
        I = self.propagate(U)
        if self.noise is not None:
            self._noise_now = torch.as_tensor(self.noise(self.it), dtype=torch.float32, device=self.dev)
        loss = self.loss(I, host_metrics=False)
        self._noise_now = None
        loss.backward()
        clean = (lambda t: torch.nan_to_num(t, nan=0.0, posinf=0.0, neginf=0.0)) if sanitize else (lambda t: t.clone())
        out = {k: clean(p.grad) for k, p in self.params.items() if p.grad is not None}
        for p in self.params.values():
            p.grad = None
        return float(loss.detach()), out

    def step(self):
        trainable = set(RAW_KEYS) if self.it >= self.warmup else set(RAW_KEYS) - {"curvature"}
        for k, p in self.params.items():
            p.grad = None
            p.requires_grad_(k in trainable)
        U = soft_window_pad(self.render(), self.pad)
        I = self.propagate(U)
        if self.noise is not None:
            self._noise_now = torch.as_tensor(self.noise(self.it), dtype=torch.float32, device=self.dev)
        loss = self.loss(I)
        self._noise_now = None
        self.last_loss = loss.item()
        loss.backward()
        tl = [self.params[k] for k in RAW_KEYS if k in trainable]
        # which Gaussians had a non-finite gradient entry this step (zeroed by nan_to_num below)
        n = self.params["pre_act_opacities"].shape[0]
        bad = torch.zeros(n, dtype=torch.bool, device=self.dev)
        for p in tl:
            bad |= ~torch.isfinite(p.grad).reshape(n, -1).all(dim=1)
        self.last_nonfinite = bad
        for p in tl:
            p.grad = torch.nan_to_num(p.grad, nan=0.0, posinf=0.0, neginf=0.0)
        torch.nn.utils.clip_grad_norm_(tl, max_norm=1.0)
        self.adan_step(trainable)
        self._sgd.step()
        self._sched.step()
        self.groups[0]["lr"] = self._sched.get_last_lr()[0]
        self.it += 1

    # -- bounded CPU sample ----------------------------------------------------------------
    def sampled_iteration_seconds(self, tile_rows=1, timer=None):
        """Seconds of one full iteration extrapolated from a bounded sample:
        splat fwd+bwd on `tile_rows` rows of 64-px tiles (scaled to all rows), BLASM fwd+bwd for one
        (plane, channel) (scaled by P*C), loss+SSIM fwd+bwd for one plane (scaled by P), and one Adan step."""
        import time
        timer = timer or time.perf_counter
        n_rows = (self.H + 63) // 64
        for p in self.params.values():
            p.grad = None
            p.requires_grad_(True)
        t0 = timer()
        h = self.render(tile_rows=(0, tile_rows))
        (h.real.sum() + h.imag.sum()).backward()
        t_render = (timer() - t0) * n_rows / tile_rows
        U = soft_window_pad(torch.polar(torch.rand(self.C, self.H, self.W, device=self.dev),
                                        torch.rand(self.C, self.H, self.W, device=self.dev)), self.pad)
        U.requires_grad_(True)
        t0 = timer()
        I = self.propagate(U, planes=[0], channels=[0])
        I.sum().backward()
        t_prop = (timer() - t0) * len(self.dist) * self.C
        I2 = torch.rand(1, self.C, self.H, self.W, device=self.dev, requires_grad=True)
        t0 = timer()
        self.loss(I2, planes=[0]).backward()
        t_loss = (timer() - t0) * len(self.dist)
        for p in self.params.values():
            if p.grad is None:
                p.grad = torch.zeros_like(p)
        t0 = timer()
        self.adan_step(set(RAW_KEYS))
        t_opt = timer() - t0
        return t_render + t_prop + t_loss + t_opt, dict(render=t_render, propagate=t_prop, loss=t_loss, adan=t_opt)
