"""Oracle: per-Gaussian preprocessing and its adjoint (numpy float64).

Test infrastructure only (see oracle/__init__.py). Restates

* Gaussians2D.apply_activations      model_2d_gaussian_rgb.py:83-112
  (grayscale twin: model_2d_gaussian_grayscale.py, lambda = wavelengths[0])
* compute_2d_covariance_elements     model_2d_gaussian_rgb.py:127-153
* invert_cov_2D                      model_2d_gaussian_rgb.py:114-125
* the CUDA-path area and radius      model_2d_gaussian_rgb.py:429-436
* the torch-path 3-sigma radius      model_2d_gaussian_rgb.py:400-403

and the hand-derived chain rule that torch autograd applies to them
(max over scales sends the gradient to the first maximal entry, the det clamp
passes the gradient where det >= 1e-10, the phase modulo has unit slope).
"""
import numpy as np

RAW_KEYS = ("means_2d", "pre_act_scales", "pre_act_rotation", "colours", "pre_act_phase", "pre_act_opacities",
            "curvature")


def _f64(a):
    return np.asarray(a, dtype=np.float64)


def activate(raw, W, H, wavelengths, pixel_pitch, curv_mode="scale_aware", eta=0.9, gray=None):
    m = _f64(raw["means_2d"])
    s_raw = _f64(raw["pre_act_scales"])
    rot = _f64(raw["pre_act_rotation"])
    ph_raw = _f64(raw["pre_act_phase"])
    o_raw = _f64(raw["pre_act_opacities"])
    c_raw = _f64(raw["curvature"])
    colours = _f64(raw["colours"])
    C = colours.shape[1]
    if gray is None:
        gray = C == 1
    t = np.tanh(m)
    means = np.stack([(t[:, 0] + 1.0) * 0.5 * W, (t[:, 1] + 1.0) * 0.5 * H], 1)
    es = np.exp(s_raw)
    scales = es + 0.1
    phase = np.mod(ph_raw, 2.0 * np.pi)
    opac = 1.0 / (1.0 + np.exp(-o_raw))
    lam = float(wavelengths[0]) if gray else float(min(wavelengths))
    dxy = float(pixel_pitch)
    arg = np.argmax(scales, axis=1)  # first maximal entry, as torch.max(dim)
    sigma = scales[np.arange(scales.shape[0]), arg]
    tc = np.tanh(c_raw)
    if curv_mode == "off":
        curv = np.zeros_like(c_raw)
        cmax = np.zeros_like(c_raw)
    elif curv_mode == "constant":
        cmax = np.full_like(c_raw, 200.0)
        curv = cmax * tc
    elif curv_mode == "scale_aware":
        cmax = eta * lam / (6.0 * sigma * dxy ** 2 + 1e-20)
        curv = cmax * tc
    else:
        raise ValueError(curv_mode)
    cr, sr = np.cos(rot), np.sin(rot)
    sx, sy = scales[:, 0], scales[:, 1]
    sx2, sy2 = sx * sx, sy * sy
    cov00 = sx2 * cr * cr + sy2 * sr * sr + 0.1
    cov01 = (sx2 - sy2) * cr * sr
    cov11 = sx2 * sr * sr + sy2 * cr * cr + 0.1
    det_raw = cov00 * cov11 - cov01 * cov01
    det = np.maximum(det_raw, 1e-10)
    inv = np.stack([cov11 / det, -cov01 / det, cov00 / det], 1)
    area = np.abs(sx * sy)
    mid = 0.5 * (cov00 + cov11)
    disc = np.sqrt(((cov00 - cov11) * 0.5) ** 2 + cov01 ** 2)
    lam_max = mid + disc
    return dict(means=means, scales=scales, rotation=rot, phase=phase, opac=opac, curv=curv, colours=colours,
                cov=np.stack([cov00, cov01, cov11], 1), inv_cov=inv, area=area,
                radii=np.ceil(5.0 * np.sqrt(lam_max)).astype(np.int32), radius3=3.0 * np.sqrt(lam_max),
                _t=t, _es=es, _arg=arg, _tc=tc, _cmax=cmax, _sigma=sigma, _det_raw=det_raw, _det=det,
                _cr=cr, _sr=sr, _lam=lam, _dxy=dxy, _mode=curv_mode, _eta=eta, _W=W, _H=H)


def activate_backward(act, g_means, g_inv, g_col, g_phase, g_opac, g_curv, g_area):
    """Chain rule from the splat-input gradients to the 7 raw parameter gradients."""
    g_means, g_inv, g_col, g_phase, g_opac, g_curv, g_area = (
        _f64(a) for a in (g_means, g_inv, g_col, g_phase, g_opac, g_curv, g_area))
    n = g_means.shape[0]
    W, H = act["_W"], act["_H"]
    t = act["_t"]
    d_m = np.stack([g_means[:, 0] * 0.5 * W * (1 - t[:, 0] ** 2), g_means[:, 1] * 0.5 * H * (1 - t[:, 1] ** 2)], 1)
    d_phase = g_phase.copy()
    o = act["opac"]
    d_o = g_opac * o * (1 - o)
    tc, cmax, sigma = act["_tc"], act["_cmax"], act["_sigma"]
    mode = act["_mode"]
    g_sigma = np.zeros(n)
    if mode == "off":
        d_c = np.zeros(n)
    elif mode == "constant":
        d_c = g_curv * 200.0 * (1 - tc ** 2)
    else:
        d_c = g_curv * cmax * (1 - tc ** 2)
        dxy = act["_dxy"]
        den = 6.0 * sigma * dxy ** 2 + 1e-20
        g_sigma = g_curv * tc * (-act["_eta"] * act["_lam"] * 6.0 * dxy ** 2 / den ** 2)
    # inverse covariance
    cov00, cov01, cov11 = act["cov"][:, 0], act["cov"][:, 1], act["cov"][:, 2]
    det, det_raw = act["_det"], act["_det_raw"]
    gi00, gi01, gi11 = g_inv[:, 0], g_inv[:, 1], g_inv[:, 2]
    g_det = -(gi00 * cov11 - gi01 * cov01 + gi11 * cov00) / det ** 2
    g_det = np.where(det_raw >= 1e-10, g_det, 0.0)
    g_c00 = gi11 / det + g_det * cov11
    g_c11 = gi00 / det + g_det * cov00
    g_c01 = -gi01 / det - 2.0 * cov01 * g_det
    # covariance -> scales, rotation
    s = act["scales"]
    sx, sy = s[:, 0], s[:, 1]
    cr, sr = act["_cr"], act["_sr"]
    g_sx = g_c00 * 2 * sx * cr * cr + g_c01 * 2 * sx * cr * sr + g_c11 * 2 * sx * sr * sr + g_area * sy
    g_sy = g_c00 * 2 * sy * sr * sr - g_c01 * 2 * sy * cr * sr + g_c11 * 2 * sy * cr * cr + g_area * sx
    g_rot = (g_c00 * 2 * cr * sr * (sy * sy - sx * sx) + g_c01 * (sx * sx - sy * sy) * (cr * cr - sr * sr)
             + g_c11 * 2 * sr * cr * (sx * sx - sy * sy))
    arg = act["_arg"]
    g_s = np.stack([g_sx, g_sy], 1)
    g_s[np.arange(n), arg] += g_sigma
    d_s = g_s * act["_es"]
    return dict(means_2d=d_m, pre_act_scales=d_s, pre_act_rotation=g_rot, colours=g_col.copy(),
                pre_act_phase=d_phase, pre_act_opacities=d_o, curvature=d_c)
