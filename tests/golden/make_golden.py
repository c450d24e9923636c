"""Generate the golden fixtures under tests/golden/ by running the reference.

This script imports the reference CVQPG Python modules from the checkout named
by --reference or by the environment variable CVQPG_REFERENCE_DIR (one of the
two is required) and records their outputs on small seeded inputs. The fixtures pin the CPU
oracle (oracle/) and the CUDA kernels to the reference's own behaviour.

Reference pieces used (paths inside the reference project):
  cuda/rasterizer.py:74-91     qpf_render_reference (uncut splat, float64 + autograd)
  model_2d_gaussian_rgb.py     Gaussians2D activations/covariance, Scene2D torch tile renderer,
  model_2d_gaussian_grayscale.py  soft_window_pad
  utils/optimizer.py           Adan (loaded by path; utils/__init__ pulls uninstalled packages)
  utils/propagator.py          propagator / multiplane_loss_odak, with the oracle's restatement of
                               the odak functions installed as the `odak` module (odak 0.2.7 is not
                               installed here, so that part stays unpinned)
  utils/data_utils.py          GaussianLoss (SSIM) with the oracle's restatement of pytorch_msssim
                               installed as `pytorch_msssim` (1.0.0 not installed: unpinned)

Run:  python tests/golden/make_golden.py [--only NAME ...]
"""
import argparse
import importlib.util
import math
import os
import sys
import types
from argparse import Namespace

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REFERENCE_DIR = os.environ.get("CVQPG_REFERENCE_DIR")  # or --reference (main)
sys.path.insert(0, REPO)


def load_by_path(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def ref(path):
    return os.path.join(REFERENCE_DIR, path)


def install_third_party_restatements():
    """Install the oracle's restatements of odak / pytorch_msssim under their import names."""
    from oracle import odak_restated, ssim as ssim_mod
    odak = types.ModuleType("odak")
    odak.pi = math.pi
    learn = types.ModuleType("odak.learn")
    wave = types.ModuleType("odak.learn.wave")
    tools = types.ModuleType("odak.learn.tools")
    for n in ("get_propagation_kernel", "generate_complex_field", "calculate_amplitude", "calculate_phase"):
        setattr(wave, n, getattr(odak_restated, n))
    for n in ("zero_pad", "crop_center", "generate_2d_gaussian"):
        setattr(tools, n, getattr(odak_restated, n))
    learn.wave, learn.tools = wave, tools
    odak.learn = learn
    sys.modules.update({"odak": odak, "odak.learn": learn, "odak.learn.wave": wave, "odak.learn.tools": tools})
    ms = types.ModuleType("pytorch_msssim")
    ms.SSIM = ssim_mod.SSIMModule
    sys.modules["pytorch_msssim"] = ms


# ---------------------------------------------------------------------------
# seeded synthetic Gaussians (activated parameters)
# ---------------------------------------------------------------------------
WAVELENGTHS = [639e-9, 515e-9, 473e-9]
PITCH = 3.74e-6


def activated_params(rng, n, W, H, C, margin=3.0):
    means = np.stack([rng.uniform(-margin, W + margin, n), rng.uniform(-margin, H + margin, n)], 1).astype(np.float32)
    s = (np.exp(rng.normal(math.log(2.0), 0.3, (n, 2))) + 0.1).astype(np.float32)
    rot = rng.uniform(0, math.pi, n).astype(np.float32)
    t = torch.from_numpy
    c, si = torch.cos(t(rot)), torch.sin(t(rot))
    sx2, sy2 = t(s[:, 0]) ** 2, t(s[:, 1]) ** 2
    cov00 = sx2 * c * c + sy2 * si * si + 0.1
    cov01 = (sx2 - sy2) * c * si
    cov11 = sx2 * si * si + sy2 * c * c + 0.1
    det = (cov00 * cov11 - cov01 * cov01).clamp(min=1e-10)
    inv = torch.stack([cov11 / det, -cov01 / det, cov00 / det], -1).numpy().astype(np.float32)
    colours = rng.uniform(0, 1, (n, C)).astype(np.float32)
    phase = rng.uniform(0, 2 * math.pi, (n, C)).astype(np.float32)
    opac = rng.uniform(0.2, 0.9, n).astype(np.float32)
    lam_min = min(WAVELENGTHS[:C]) if C == 3 else WAVELENGTHS[0]
    cmax = 0.9 * lam_min / (6.0 * s.max(1) * PITCH ** 2)
    curv = (cmax * np.tanh(rng.normal(0, 1, n))).astype(np.float32)
    area = np.abs(s[:, 0] * s[:, 1]).astype(np.float32)
    wl = WAVELENGTHS if C == 3 else WAVELENGTHS[:1]
    k = (2 * np.pi / torch.tensor(wl, dtype=torch.float32)).numpy().astype(np.float32)
    dxy2 = np.float32(PITCH ** 2)
    cov = np.stack([cov00.numpy(), cov01.numpy(), cov11.numpy()], 1).astype(np.float32)
    return dict(means=means, inv_cov=inv, colours=colours, phase=phase, opac=opac, curv=curv, area=area, k=k,
                dxy2=dxy2, cov=cov)


# ---------------------------------------------------------------------------
# fixtures
# ---------------------------------------------------------------------------
def golden_splat(C, name, seed, n=200, W=50, H=40):
    rasterizer = load_by_path("ref_cuda_rasterizer", ref("cuda/rasterizer.py"))
    rng = np.random.default_rng(seed)
    p = activated_params(rng, n, W, H, C)
    T = lambda a: torch.from_numpy(np.asarray(a, dtype=np.float64)).requires_grad_(True)
    ins = [T(p[k]) for k in ("means", "inv_cov", "colours", "phase", "opac", "curv", "area")]
    out = rasterizer.qpf_render_reference(*ins, torch.from_numpy(p["k"].astype(np.float64)), float(p["dxy2"]), W, H)
    gw = rng.normal(0, 1, (C, H, W)) + 1j * rng.normal(0, 1, (C, H, W))
    loss = (out.real * torch.from_numpy(gw.real)).sum() + (out.imag * torch.from_numpy(gw.imag)).sum()
    loss.backward()
    grads = {f"d_{k}": t.grad.numpy() for k, t in zip(("means", "inv_cov", "colours", "phase", "opac", "curv", "area"),
                                                       ins)}
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), W=W, H=H, grad_field=gw, out=out.detach().numpy(),
                        **p, **grads)


def _args_prop(C, pad_size, renderer="torch", phase_iso=False):
    wl = WAVELENGTHS if C == 3 else WAVELENGTHS[:1]
    return Namespace(wavelengths=list(wl), pixel_pitch=PITCH, pad_size=list(pad_size), tile_size=64, gauss_batch=1024,
                     phase_iso=phase_iso, grad_ckpt=False, renderer=renderer, curv_nyquist=0.9)


def raw_params(rng, n, W, H, C, curv_scale=1.0):
    """Raw (pre-activation) parameters in the Gaussians2D layout (model_2d_gaussian_rgb.py:18-26)."""
    mx = rng.uniform(0, W, n) / W * 2 - 1
    my = rng.uniform(0, H, n) / H * 2 - 1
    means = np.arctanh(np.clip(np.stack([mx, my], 1), -0.999, 0.999)).astype(np.float32)
    scales = np.log(np.exp(rng.normal(math.log(2.0), 0.3, (n, 2)))).astype(np.float32)
    rot = rng.uniform(-math.pi, math.pi, n).astype(np.float32)
    colours = rng.uniform(0, 1, (n, C)).astype(np.float32)
    phase = rng.uniform(-1.0, 7.5, (n, C)).astype(np.float32)   # exercises the mod-2pi wrap
    opac = rng.normal(-0.5, 1.0, n).astype(np.float32)
    curv = (curv_scale * rng.normal(0, 0.5, n)).astype(np.float32)
    return dict(means_2d=means, pre_act_scales=scales, pre_act_rotation=rot, colours=colours,
                pre_act_phase=phase, pre_act_opacities=opac, curvature=curv)


RAW_KEYS = ("means_2d", "pre_act_scales", "pre_act_rotation", "colours", "pre_act_phase", "pre_act_opacities",
            "curvature")


def _make_gaussians(model, raw, W, H, C, args_prop, curv_mode):
    g = model.Gaussians2D(num_points=raw["means_2d"].shape[0], img_size=(W, H), device="cpu", args_prop=args_prop)
    for k in RAW_KEYS:
        getattr(g, k).data.copy_(torch.from_numpy(raw[k]))
    g.curv_mode = curv_mode
    model.make_trainable_2d(g)
    return g


def golden_preprocess(C, name, seed, n=300, W=96, H=80):
    model = load_by_path(f"ref_model_{C}", ref("model_2d_gaussian_rgb.py" if C == 3 else
                                              "model_2d_gaussian_grayscale.py"))
    rng = np.random.default_rng(seed)
    raw = raw_params(rng, n, W, H, C)
    raw["pre_act_scales"][:5, 0] = raw["pre_act_scales"][:5, 1]  # ties in max(scales)
    out = {}
    for mode in ("scale_aware", "constant", "off"):
        g = _make_gaussians(model, raw, W, H, C, _args_prop(C, (H + 32, W + 32)), mode)
        scales, rotation, phase, opac, means, curv = g.apply_activations()
        c00, c01, c11 = g.compute_2d_covariance_elements(scales, rotation)
        i00, i01, i11 = g.invert_cov_2D(c00, c01, c11)
        area = (scales[:, 0] * scales[:, 1]).abs()
        with torch.no_grad():
            mid = 0.5 * (c00 + c11)
            disc = torch.sqrt(((c00 - c11) * 0.5) ** 2 + c01 ** 2)
            radii = (5.0 * torch.sqrt(mid + disc)).ceil().to(torch.int32)
            radius3 = 3.0 * torch.sqrt(mid + disc)
        outs = dict(means=means, inv_cov=torch.stack([i00, i01, i11], -1), phase=phase, opac=opac, curv=curv,
                    area=area, cov=torch.stack([c00, c01, c11], -1))
        rng2 = np.random.default_rng(seed + 1)
        wts = {k: torch.from_numpy(rng2.normal(0, 1, v.shape).astype(np.float32)) for k, v in outs.items()
               if k != "cov"}
        loss = sum((v * wts[k]).sum() for k, v in outs.items() if k != "cov")
        loss.backward()
        for k, v in outs.items():
            out[f"{mode}__{k}"] = v.detach().numpy()
        for k, v in wts.items():
            out[f"{mode}__w_{k}"] = v.numpy()
        out[f"{mode}__radii"] = radii.numpy()
        out[f"{mode}__radius3"] = radius3.numpy()
        for k in RAW_KEYS:
            gr = getattr(g, k).grad
            out[f"{mode}__grad_{k}"] = np.zeros(raw[k].shape, np.float32) if gr is None else gr.numpy()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), W=W, H=H, C=C, **raw, **out)


def golden_torch_renderer(C, name, seed, n=400, W=160, H=112, pad=(176, 224), phase_iso=False):
    """The reference torch tile renderer (3-sigma 64-px culling) + soft_window_pad, with gradients.

    phase_iso=True renders the isotropic quadratic phase of --phase_iso."""
    model = load_by_path(f"ref_model_{C}", ref("model_2d_gaussian_rgb.py" if C == 3 else
                                              "model_2d_gaussian_grayscale.py"))
    rng = np.random.default_rng(seed)
    raw = raw_params(rng, n, W, H, C, curv_scale=2.0)
    ap = _args_prop(C, pad, phase_iso=phase_iso)
    g = _make_gaussians(model, raw, W, H, C, ap, "scale_aware")
    with torch.no_grad():
        scales, rotation, phase, opac, means, curv = g.apply_activations()
        c00, c01, c11 = g.compute_2d_covariance_elements(scales, rotation)
        i00, i01, i11 = g.invert_cov_2D(c00, c01, c11)
        mid = 0.5 * (c00 + c11)
        disc = torch.sqrt(((c00 - c11) * 0.5) ** 2 + c01 ** 2)
        act = dict(act_means=means.numpy(), act_inv_cov=torch.stack([i00, i01, i11], -1).numpy(),
                   act_phase=phase.numpy(), act_opac=opac.numpy(), act_curv=curv.numpy(),
                   act_area=(scales[:, 0] * scales[:, 1]).abs().numpy(), act_radius3=(3.0 * torch.sqrt(mid + disc)).numpy(),
                   act_radii=(5.0 * torch.sqrt(mid + disc)).ceil().to(torch.int32).numpy(),
                   act_k=(2 * np.pi / torch.tensor(ap.wavelengths, dtype=torch.float32)).numpy(),
                   act_dxy2=np.float32(ap.pixel_pitch ** 2))
    g.invalidate_cache()
    scene = model.Scene2D(g, ap)
    saved = model.soft_window_pad
    model.soft_window_pad = lambda h, p: h
    try:
        field = scene.render((W, H))
    finally:
        model.soft_window_pad = saved
    padded = saved(field, ap.pad_size)
    gw = torch.from_numpy((rng.normal(0, 1, padded.shape) + 1j * rng.normal(0, 1, padded.shape)).astype(np.complex64))
    loss = (padded.real * gw.real).sum() + (padded.imag * gw.imag).sum()
    loss.backward()
    grads = {f"grad_{k}": getattr(g, k).grad.numpy() for k in RAW_KEYS}
    # field-level gradient of the same loss through the pad (for the pad adjoint)
    f2 = field.detach().clone().requires_grad_(True)
    l2 = (saved(f2, ap.pad_size).real * gw.real).sum() + (saved(f2, ap.pad_size).imag * gw.imag).sum()
    l2.backward()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), W=W, H=H, C=C, pad=np.array(pad), **raw,
                        field=field.detach().numpy(), padded=padded.detach().numpy(), grad_padded=gw.numpy(),
                        grad_field=f2.grad.numpy(), **grads, **act)


def golden_propagate(C, name, seed, H, W, pH, pW, P, d_val, vd, aperture_size):
    """soft_window_pad -> phase/amplitude -> propagator.reconstruct -> crop (train_2d_gaussian_rgb.py:89-95, 193)."""
    model = load_by_path(f"ref_model_{C}", ref("model_2d_gaussian_rgb.py" if C == 3 else
                                              "model_2d_gaussian_grayscale.py"))
    prop_mod = load_by_path("ref_propagator", ref("utils/propagator.py"))
    import odak
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.0, 1.35, (C, H, W))
    field = (amp * np.exp(1j * rng.uniform(0, 2 * np.pi, (C, H, W)))).astype(np.complex64)
    field[0, 3, 5] = 0.0  # exact zero: the clamp/angle adjoint returns 0 there
    wl = WAVELENGTHS if C == 3 else WAVELENGTHS[:1]
    distances = torch.linspace(-vd / 2.0, vd / 2.0, P) + d_val if P > 1 else torch.tensor([d_val])
    prop = prop_mod.propagator(resolution=[pH, pW], wavelengths=wl, pixel_pitch=PITCH, number_of_frames=C,
                               distances=distances, propagation_type="Bandlimited Angular Spectrum",
                               laser_channel_power=torch.eye(C), aperture_size=aperture_size, device="cpu")
    f = torch.from_numpy(field).requires_grad_(True)
    U = model.soft_window_pad(f, [pH, pW])
    phase = odak.learn.wave.calculate_phase(U) % (2 * odak.pi)
    amplitude = torch.clamp(odak.learn.wave.calculate_amplitude(U), min=0.0, max=1.0)
    rec = prop.reconstruct(phase, amplitude=amplitude, no_grad=False)
    I_full = torch.sum(rec, dim=0)
    I_crop = odak.learn.tools.crop_center(I_full, size=(H, W))
    wts = torch.from_numpy(rng.normal(0, 1, (P, C, H, W)).astype(np.float32))
    (I_crop * wts).sum().backward()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), field=field, H=H, W=W, pH=pH, pW=pW,
                        distances=distances.double().numpy(), wavelengths=np.array(wl), pitch=PITCH,
                        aperture=float(aperture_size), I_full=I_full.detach().numpy(),
                        I_crop=I_crop.detach().numpy(), wts=wts.numpy(), grad_field=f.grad.numpy())


class _MeansCosine:
    """The training script's MeansCosineScheduler (train_2d_gaussian_rgb.py:58-70), restated as glue
    because the script itself imports packages that are not installed here."""

    def __init__(self, optimizer, num_itrs, eta_min=1e-3):
        self.optimizer = optimizer
        self.group_indices = [i for i, g in enumerate(optimizer.param_groups) if g.get("name") == "means"]
        tmp = torch.optim.SGD([{"params": optimizer.param_groups[i]["params"], "lr": optimizer.param_groups[i]["lr"]}
                               for i in self.group_indices])
        self.sch = torch.optim.lr_scheduler.CosineAnnealingLR(tmp, T_max=max(1, num_itrs), eta_min=eta_min)

    def step(self):
        self.sch.step()
        for i, gi in enumerate(self.group_indices):
            self.optimizer.param_groups[gi]["lr"] = self.sch.get_last_lr()[i]


def golden_targets(C, name, seed, H=72, W=104, P=4):
    """Multi-plane defocus targets of the reference loss (utils/propagator.py:361-415) via get_targets()."""
    from complex_valued_quadratic_phase_gaussian_b200 import scenes as sc
    prop_mod = load_by_path("ref_propagator", ref("utils/propagator.py"))
    img, depth = sc.rgb_blobs(H, W, seed=seed, num_blobs=60) if C == 3 else sc.grayscale_blobs(H, W, seed=seed)
    img = img.copy()
    img[:, :, :6] = 0.0   # a zero column band: exercises planes whose masked image sums to zero
    depth = 0.8 * depth  # planes 0..2 over the scene
    depth[:, :6] = 0.99   # ... and plane 3 only on the zero band, so its masked image sums to zero
    loss_fn = prop_mod.multiplane_loss_odak(target_image=torch.from_numpy(img),
                                            target_depth=torch.from_numpy(depth)[None], target_blur_size=20,
                                            number_of_planes=P, blur_ratio=8, weights=[1.0, 1.0, 1.0, 0.0],
                                            scheme="defocus", reduction="mean", split_ratio=1.0, device="cpu")
    targets, masks, qdepth = loss_fn.get_targets()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), image=img, depth=depth, P=P,
                        targets=targets.numpy().astype(np.float32),
                        plane=np.rint(qdepth.numpy().reshape(H, W) * (P - 1)).astype(np.uint8))


def golden_fit(C, name, seed, W=96, H=64, N=200, P=2, pad=(96, 128), iters=3, warmup=1, num_itrs=10,
               d_val=1e-3, vd=1e-3):
    """Iterations of the reference fit loop body (train_2d_gaussian_rgb.py:179-211) on the torch renderer."""
    from oracle import loss as oloss
    from complex_valued_quadratic_phase_gaussian_b200 import scenes as sc
    model = load_by_path(f"ref_model_{C}", ref("model_2d_gaussian_rgb.py" if C == 3 else
                                              "model_2d_gaussian_grayscale.py"))
    prop_mod = load_by_path("ref_propagator", ref("utils/propagator.py"))
    opt_mod = load_by_path("ref_optimizer", ref("utils/optimizer.py"))
    du = load_by_path("ref_data_utils", ref("utils/data_utils.py"))
    import odak
    torch.manual_seed(seed)
    if C == 3:
        img, depth = sc.rgb_blobs(H, W, seed=seed, num_blobs=40)
    else:
        img, depth = sc.grayscale_blobs(H, W, seed=seed, num_blobs=12)
    wl = WAVELENGTHS if C == 3 else WAVELENGTHS[:1]
    ap = _args_prop(C, pad)
    ap.num_planes, ap.split_ratio = P, 1.0
    distances = torch.linspace(-vd / 2.0, vd / 2.0, P) + d_val
    prop = prop_mod.propagator(resolution=list(pad), wavelengths=wl, pixel_pitch=PITCH, number_of_frames=C,
                               distances=distances, propagation_type="Bandlimited Angular Spectrum",
                               laser_channel_power=torch.eye(C), aperture_size=10 * max(W, H), device="cpu")
    loss_fn = prop_mod.multiplane_loss_odak(target_image=torch.from_numpy(img), target_depth=torch.from_numpy(depth)[None],
                                            target_blur_size=20, number_of_planes=P, blur_ratio=8,
                                            weights=[1.0, 1.0, 1.0, 0.0], scheme="defocus", reduction="mean",
                                            split_ratio=1.0, device="cpu")
    targets, masks, qdepth = loss_fn.get_targets()
    rng = np.random.default_rng(seed)
    raw = raw_params(rng, N, W, H, C, curv_scale=1.0)
    raw["pre_act_phase"] = rng.uniform(0, 2 * np.pi, (N, C)).astype(np.float32)
    g = _make_gaussians(model, raw, W, H, C, ap, "scale_aware")
    scene = model.Scene2D(g, ap)
    g.curvature.requires_grad_(False)
    groups = [{"params": [g.means_2d], "lr": 0.01, "name": "means"},
              {"params": [g.pre_act_scales], "lr": 0.005, "name": "scales"},
              {"params": [g.colours, g.pre_act_phase], "lr": 0.0025, "name": "amplitude_phase"},
              {"params": [g.pre_act_opacities], "lr": 0.025, "name": "opacity"},
              {"params": [g.pre_act_rotation], "lr": 0.001, "name": "rotation"},
              {"params": [g.curvature], "lr": 0.001, "name": "curvature"}]
    opt = opt_mod.Adan(groups, lr=0, eps=1e-8, foreach=False)
    sched = _MeansCosine(opt, num_itrs)
    trainable = [p for gr in groups for p in gr["params"]]
    rec = {"loss": [], "mse0": []}
    noise_seed = seed
    real_randn_like = torch.randn_like
    for itr in range(iters):
        if itr == warmup:
            g.curvature.requires_grad_(True)
        opt.zero_grad()
        holo = scene.render((W, H))
        phase_map = odak.learn.wave.calculate_phase(holo) % (2 * odak.pi)
        amp = torch.clamp(odak.learn.wave.calculate_amplitude(holo), min=0.0, max=1.0)
        recon = prop.reconstruct(phase_map, amplitude=amp, no_grad=False).sum(0)
        noise = torch.from_numpy(oloss.plane_noise((P, C, H, W), noise_seed, itr))
        loss = 0.0
        for idx, (ri, tgt) in enumerate(zip(recon, targets)):
            pred = torch.clamp(odak.learn.tools.crop_center(ri, size=(H, W)), min=0.0, max=1.0)
            torch.randn_like = lambda t, _n=noise[idx]: _n.clone()
            try:
                loss = loss + loss_fn(pred, tgt, idx, inject_noise=True)
            finally:
                torch.randn_like = real_randn_like
            loss = loss + (du.GaussianLoss(pred, tgt) if C == 3 else du.GaussianLossGrayscale(pred, tgt))
            if idx == 0:
                rec["mse0"].append(float(((pred - tgt) ** 2).mean()))
        rec["loss"].append(float(loss))
        loss.backward()
        for p_ in trainable:
            if p_.grad is not None:
                p_.grad = torch.nan_to_num(p_.grad, nan=0.0, posinf=0.0, neginf=0.0)
        torch.nn.utils.clip_grad_norm_(trainable, max_norm=1.0)
        opt.step()
        sched.step()
        for k in RAW_KEYS:
            rec.setdefault(f"it{itr}_{k}", getattr(g, k).detach().numpy().copy())
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), W=W, H=H, C=C, N=N, P=P, pad=np.array(pad),
                        distances=distances.double().numpy(), wavelengths=np.array(wl), pitch=PITCH, seed=noise_seed,
                        warmup=warmup, num_itrs=num_itrs, iters=iters, aperture=10 * max(W, H),
                        targets=targets.numpy(),
                        depth_plane=loss_fn.target_depth.numpy().astype(np.uint8).reshape(H, W),  # plane index
                        loss=np.array(rec["loss"]), mse0=np.array(rec["mse0"]),
                        **{f"init_{k}": v for k, v in raw.items()},
                        **{k: v for k, v in rec.items() if k.startswith("it")})


def golden_checkpoint(name="checkpoint", seed=71, n=50, W=40, H=24, C=3):
    """Checkpoint format both ways: the reference's Gaussians2D.save_gaussians writes
    checkpoint_ref.pth (model_2d_gaussian_rgb.py:155-167), and a checkpoint written by this
    library's save_gaussians is read back by the reference's load_gaussians (:169-180); what the
    reference loaded is recorded."""
    import tempfile
    from complex_valued_quadratic_phase_gaussian_b200.fit import save_gaussians
    model = load_by_path(f"ref_model_{C}", ref("model_2d_gaussian_rgb.py"))
    rng = np.random.default_rng(seed)
    raw = raw_params(rng, n, W, H, C)
    g = _make_gaussians(model, raw, W, H, C, _args_prop(C, (H + 32, W + 32)), "scale_aware")
    g.save_gaussians(os.path.join(HERE, f"{name}_ref.pth"))
    raw2 = raw_params(np.random.default_rng(seed + 1), n, W, H, C)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "ours.pth")
        save_gaussians(raw2, (W, H), path)
        g2 = model.Gaussians2D(num_points=n, img_size=(W, H), device="cpu", args_prop=_args_prop(C, (H + 32, W + 32)))
        g2.load_gaussians(path)
        loaded = {f"loaded_{k}": getattr(g2, k).detach().numpy().copy() for k in RAW_KEYS}
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), W=W, H=H, C=C, **{f"ref_{k}": v for k, v in raw.items()},
                        **{f"ours_{k}": v for k, v in raw2.items()}, **loaded)


def golden_dpac(name="dpac", seed=81, C=3, W=40, H=28, pad=(64, 72)):
    """The reference's POH encoding (export_poh.py:110-119, 175-180): soft_window_pad of a splat
    field (model_2d_gaussian_rgb.py:186-241), phase mod 2 pi, amplitude clamped to 1, dpac(),
    round(poh / 2 pi * 256) mod 256. export_poh.py is loaded by path; its evaluation-only imports
    (lpips, pycvvdp: not installed) are empty stand-ins, never called here."""
    import odak
    for mod in ("lpips", "pycvvdp"):
        sys.modules.setdefault(mod, types.ModuleType(mod))
    model = load_by_path(f"ref_model_{C}", ref("model_2d_gaussian_rgb.py"))
    exp = load_by_path("ref_export_poh", ref("export_poh.py"))
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.0, 1.4, (C, H, W))  # some amplitudes above 1: the clamp acts
    field = (amp * np.exp(1j * rng.uniform(-np.pi, np.pi, (C, H, W)))).astype(np.complex64)
    padded = model.soft_window_pad(torch.from_numpy(field), list(pad))
    phase = odak.learn.wave.calculate_phase(padded) % (2 * np.pi)
    amplitude = odak.learn.wave.calculate_amplitude(padded).clamp(0.0, 1.0)
    levels = torch.round(exp.dpac(phase, amplitude) / (2 * np.pi) * 256).to(torch.int64) % 256
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), field=field, pad=np.array(pad),
                        levels=levels.numpy().astype(np.uint8))


GOLDENS = {
    "splat_rgb": lambda: golden_splat(3, "splat_rgb", 11),
    "splat_gray": lambda: golden_splat(1, "splat_gray", 12),
    "preprocess_rgb": lambda: golden_preprocess(3, "preprocess_rgb", 21),
    "preprocess_gray": lambda: golden_preprocess(1, "preprocess_gray", 22),
    "torch_renderer_rgb": lambda: golden_torch_renderer(3, "torch_renderer_rgb", 31),
    "torch_renderer_gray": lambda: golden_torch_renderer(1, "torch_renderer_gray", 32),
    "torch_renderer_iso_rgb": lambda: golden_torch_renderer(3, "torch_renderer_iso_rgb", 33, phase_iso=True),
    # 2pH = 176 = 16*11, 2pW = 208 = 16*13, 3 planes, aperture wide open (train default 10*max(img))
    "propagate_rgb": lambda: golden_propagate(3, "propagate_rgb", 41, 40, 56, 88, 104, 3, 1e-3, 1e-3, 560),
    # 2pH = 2pW = 120 = 8*3*5: band limit active (z = 5 cm) and a small Fourier aperture
    "propagate_gray_bandlimit": lambda: golden_propagate(1, "propagate_gray_bandlimit", 42, 32, 32, 60, 60, 2,
                                                         5e-2, 2e-2, 40),
    "targets_rgb": lambda: golden_targets(3, "targets_rgb", 61),
    "fit_rgb": lambda: golden_fit(3, "fit_rgb", 51),
    "fit_gray": lambda: golden_fit(1, "fit_gray", 52, P=3),
    "checkpoint": lambda: golden_checkpoint(),
    "dpac": lambda: golden_dpac(),
}


def main():
    global REFERENCE_DIR
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", default=None)
    ap.add_argument("--reference", default=REFERENCE_DIR,
                    help="the reference checkout (default: the CVQPG_REFERENCE_DIR environment variable)")
    a = ap.parse_args()
    REFERENCE_DIR = a.reference
    if not REFERENCE_DIR or not os.path.isdir(REFERENCE_DIR):
        raise SystemExit(f"reference checkout not found ({REFERENCE_DIR!r}): pass --reference or set "
                         "CVQPG_REFERENCE_DIR")
    torch.set_num_threads(8)
    install_third_party_restatements()
    for name, fn in GOLDENS.items():
        if a.only and name not in a.only:
            continue
        print("golden:", name, flush=True)
        fn()


if __name__ == "__main__":
    main()
