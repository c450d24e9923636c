"""GPU: the preprocessing kernels (activations, covariance, inverse, radii and their adjoint)
through the C-ABI, against the reference's own outputs (tests/golden/preprocess_*.npz, made by
Gaussians2D.apply_activations / compute_2d_covariance_elements / invert_cov_2D and torch autograd,
model_2d_gaussian_rgb.py:83-153) in all three curvature modes.

Gates: activated values within 1e-6 relative L2 (1e-5 for the inverse covariance, whose
determinant cancels), radii bit-exact, the 3-sigma radius within 8 ulp, tile counts equal to the oracle's, raw-parameter gradients
within 1e-5 relative L2 of torch autograd.
"""
import ctypes

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu
RAW = ("means_2d", "pre_act_scales", "pre_act_rotation", "colours", "pre_act_phase", "pre_act_opacities",
       "curvature")
MODES = {"off": 0, "constant": 1, "scale_aware": 2}


class PreParams(ctypes.Structure):
    _fields_ = [("channels", ctypes.c_int), ("num_gaussians", ctypes.c_int), ("width", ctypes.c_int),
                ("height", ctypes.c_int), ("curv_mode", ctypes.c_int), ("curv_trainable", ctypes.c_int),
                ("warmup_iters", ctypes.c_int), ("pixel_pitch", ctypes.c_double),
                ("wavelengths", ctypes.c_double * 3), ("curv_nyquist", ctypes.c_double),
                ("curv_const", ctypes.c_double)]


def _params(g, mode):
    C, N = int(g["C"]), int(g["means_2d"].shape[0])
    p = PreParams()
    p.channels, p.num_gaussians, p.width, p.height = C, N, int(g["W"]), int(g["H"])
    p.curv_mode, p.curv_trainable, p.warmup_iters = MODES[mode], 1, 0
    p.pixel_pitch = 3.74e-6
    wl = [639e-9, 515e-9, 473e-9] if C == 3 else [639e-9, 0.0, 0.0]
    for i in range(3):
        p.wavelengths[i] = wl[i]
    p.curv_nyquist, p.curv_const = 0.9, 200.0
    return p


def _flat(g):
    return torch.from_numpy(np.concatenate([g[k].astype(np.float32).ravel() for k in RAW])).cuda()


@pytest.mark.parametrize("name", ["preprocess_rgb", "preprocess_gray"])
@pytest.mark.parametrize("mode", ["scale_aware", "constant", "off"])
def test_preprocess_kernels_match_reference(golden, name, mode):
    from complex_valued_quadratic_phase_gaussian_b200 import _lib
    lib = _lib.lib()
    g = golden(name)
    C, N = int(g["C"]), int(g["means_2d"].shape[0])
    p = _params(g, mode)
    flat = _flat(g)
    rec = torch.zeros(N, 16, dtype=torch.float32, device="cuda")
    radii = torch.zeros(N, dtype=torch.int32, device="cuda")
    r3 = torch.zeros(N, dtype=torch.float32, device="cuda")
    tiles = torch.zeros(N, dtype=torch.int32, device="cuda")
    s = _lib.stream_of(torch.device("cuda"))
    _lib.check(lib.cvqpg_preprocess_forward(ctypes.byref(p), _lib.ptr(flat), _lib.ptr(rec), _lib.ptr(radii),
                                            _lib.ptr(r3), _lib.ptr(tiles), s), "cvqpg_preprocess_forward")
    r = rec.cpu().numpy().astype(np.float64)
    got = {"means": r[:, 0:2], "inv_cov": r[:, 2:5], "opac": r[:, 5], "curv": r[:, 6], "area": r[:, 7],
           "phase": r[:, 8 + C:8 + 2 * C]}
    for key, v in got.items():
        ref = g[f"{mode}__{key}"].astype(np.float64)
        if key == "curv" and mode == "off":
            assert np.all(v == 0) and np.all(ref == 0)
            continue
        tol = 1e-5 if key == "inv_cov" else 1e-6
        assert rel_l2(v, ref) < tol, (key, rel_l2(v, ref))
    np.testing.assert_array_equal(r[:, 8:8 + C], g["colours"])
    assert np.array_equal(radii.cpu().numpy(), g[f"{mode}__radii"])
    # the float32 covariance differs from torch's CPU one by an ulp where the GPU contracts a
    # product and a sum into one FMA; 3 sqrt(lambda_max) inherits that (the integer radii match)
    ref3 = g[f"{mode}__radius3"]
    d3 = np.abs(r3.cpu().numpy().astype(np.float64) - ref3) / np.spacing(ref3)
    print(f"{name} {mode}: radius3 max {d3.max():.1f} ulp from the reference")
    assert d3.max() <= 8
    from oracle import splat as osp
    _, lgx, lgy = osp.list_grid(osp.CULL_CUDA16_5SIGMA, int(g["W"]), int(g["H"]))
    expect = [len(osp._tiles_of(i, osp.CULL_CUDA16_5SIGMA, got["means"].astype(np.float32), int(g["W"]), int(g["H"]),
                                g[f"{mode}__radii"], None, lgx, lgy)) for i in range(N)]
    assert np.array_equal(tiles.cpu().numpy(), np.array(expect))

    # adjoint: the golden's upstream weights as the splat gradients (colours get none)
    w = {k: g[f"{mode}__w_{k}"].astype(np.float32) for k in ("means", "inv_cov", "phase", "opac", "curv", "area")}
    sg = np.concatenate([w["means"].ravel(), w["inv_cov"].ravel(), np.zeros(N * C, np.float32), w["phase"].ravel(),
                         w["opac"], w["curv"], w["area"]])
    sg_d = torch.from_numpy(sg).cuda()
    grads = torch.zeros_like(flat)
    partials = torch.zeros(int(lib.cvqpg_preprocess_partials(N)), dtype=torch.float32, device="cuda")
    _lib.check(lib.cvqpg_preprocess_backward(ctypes.byref(p), _lib.ptr(flat), _lib.ptr(sg_d), _lib.ptr(grads), None,
                                             _lib.ptr(partials), s), "cvqpg_preprocess_backward")
    gr = grads.cpu().numpy().astype(np.float64)
    off = 0
    for k in RAW:
        n = g[k].size
        ref = g[f"{mode}__grad_{k}"].astype(np.float64).ravel()
        mine = gr[off:off + n]
        off += n
        if np.linalg.norm(ref) == 0:
            assert np.all(mine == 0), k
        else:
            assert rel_l2(mine, ref) < 1e-5, (k, rel_l2(mine, ref))
    # the clip's sum of squares covers every gradient
    assert abs(float(partials.sum()) - float((gr ** 2).sum())) <= 1e-5 * float((gr ** 2).sum())
