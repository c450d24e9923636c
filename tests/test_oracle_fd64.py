"""CPU: pin the float64 finite-difference checker (oracle/fd64.py) to the numpy oracle:
its loss equals the oracle's noise-free fit loss, a perturbed Gaussian's loss equals the
oracle's at the same tile lists, and its central differences match the oracle's analytic
raw-parameter gradient."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import blasm as ob
from oracle import fd64
from oracle import loss as ol
from oracle import preprocess as opre
from oracle import splat as osp

RAW = opre.RAW_KEYS


def _scene(seed=5, W=64, H=48, N=60, P=2, pad=(80, 96)):
    from complex_valued_quadratic_phase_gaussian_b200 import scenes as sc
    from complex_valued_quadratic_phase_gaussian_b200.fit import FitConfig, synthetic_init
    img, depth = sc.grayscale_blobs(H, W, seed=seed, num_blobs=8)
    targets, q = ol.defocus_targets(img, depth, P)
    cfg = FitConfig(img_size=(W, H), num_gaussians=N, wavelengths=[515e-9], pixel_pitch=8e-6, num_planes=P,
                    d_val=1.5e-3, volume_depth=1e-3, pad_size=list(pad), seed=seed)
    raw = {k: v.numpy().astype(np.float64) for k, v in synthetic_init(cfg, seed).items()}
    return cfg, raw, targets, q


def _checker(cfg, raw, targets, q):
    return fd64.FiniteDifferenceLoss(raw, cfg.W, cfg.H, cfg.wavelengths, cfg.pixel_pitch, cfg.resolved_pad(),
                                     cfg.distances(), cfg.resolved_aperture(), targets, q)


def _oracle_loss(cfg, act, pl, ranges, targets, q):
    k = (np.float32(2 * np.pi) / np.asarray(cfg.wavelengths, dtype=np.float32)).astype(np.float64)
    dxy2 = float(np.float32(cfg.pixel_pitch ** 2))
    U = osp.splat_forward(act["means"], act["inv_cov"], act["colours"], act["phase"], act["opac"], act["curv"],
                          act["area"], k, dxy2, cfg.W, cfg.H, cull=osp.CULL_CUDA16_5SIGMA, point_list=pl,
                          ranges=ranges)
    pH, pW = cfg.resolved_pad()
    V = ob.chain_forward(U, pH, pW, cfg.wavelengths, cfg.distances(), cfg.pixel_pitch,
                         aperture_radius=cfg.resolved_aperture())
    return ol.multiplane_loss(V, targets, q)[0], U, V


def test_loss_matches_oracle_and_perturbation_keeps_lists():
    cfg, raw, targets, q = _scene(W=112, H=96, N=40, pad=(128, 144))
    fd = _checker(cfg, raw, targets, q)
    base, _, _ = _oracle_loss(cfg, fd.act, fd.pl, fd.ranges, targets, q)
    assert abs(fd.base_loss() - base) < 1e-12 * abs(base)
    a = fd.act
    inside = [i for i in range(a["means"].shape[0]) if a["radii"][i] + 16 < a["means"][i, 0] < cfg.W - a["radii"][i] - 16
              and a["radii"][i] + 16 < a["means"][i, 1] < cfg.H - a["radii"][i] - 16]
    g = inside[0]  # its tiles stay inside the image, so the guard band does not move
    for key, idx in (("pre_act_scales", 1), ("curvature", None), ("means_2d", 0)):
        pert = {k: v.copy() for k, v in raw.items()}
        if idx is None:
            pert[key][g] += 0.01
            val = pert[key][g]
        else:
            pert[key][g, idx] += 0.01
            val = pert[key][g, idx]
        act = opre.activate(pert, cfg.W, cfg.H, cfg.wavelengths, cfg.pixel_pitch)
        ref, _, _ = _oracle_loss(cfg, act, fd.pl, fd.ranges, targets, q)  # g's support stays off the edges
        assert abs(fd.loss_with(g, key, idx, val) - ref) < 1e-11 * abs(ref), key


def test_central_differences_match_oracle_adjoint():
    cfg, raw, targets, q = _scene()
    fd = _checker(cfg, raw, targets, q)
    _, U, V = _oracle_loss(cfg, fd.act, fd.pl, fd.ranges, targets, q)
    _, _, _, gV = ol.multiplane_loss(V, targets, q)
    pH, pW = cfg.resolved_pad()
    gU = ob.chain_backward(U, gV, pH, pW, cfg.wavelengths, cfg.distances(), cfg.pixel_pitch,
                           aperture_radius=cfg.resolved_aperture())
    a = fd.act
    gs = osp.splat_backward(gU, a["means"], a["inv_cov"], a["colours"], a["phase"], a["opac"], a["curv"], a["area"],
                            fd.k, fd.dxy2, cfg.W, cfg.H, cull=osp.CULL_CUDA16_5SIGMA, point_list=fd.pl,
                            ranges=fd.ranges)
    grads = opre.activate_backward(a, *gs)
    fds, ans = [], []
    for g in (3, 11, 29):
        for key in RAW:
            for idx in (tuple(range(raw[key].shape[1])) if raw[key].ndim == 2 else (None,)):
                fds.append(fd.central_difference(g, key, idx, h=1e-4))
                ans.append(grads[key][g] if idx is None else grads[key][g, idx])
    assert rel_l2(fds, ans) < 1e-6, rel_l2(fds, ans)
