"""Phase-only hologram (POH) export of a fit, as the reference's export_poh.py does it.

``export_poh(fitter)``: the fit's field -> soft window pad + amplitude clamp ->
DPAC -> 8-bit levels [C, pH, pW] (cvqpg_poh_encode, one kernel), then the
reconstruction of the 8-bit hologram through a Fourier aperture of radius
min(W, H) (the reference default) to every plane (the propagation with
input_mode 1), cropped to the image, and its per-plane PSNR against the fit's
targets. The reference writes PNGs; here the levels stay a uint8 tensor.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .propagator import BlasmPlan


def export_poh(fitter, aperture_size=None):
    cfg = fitter.cfg
    C, H, W, P = fitter.C, fitter.H, fitter.W, fitter.P
    pH, pW = cfg.resolved_pad()
    dev = fitter.device
    field = torch.empty((C, H, W), dtype=torch.complex64, device=dev)
    fitter.evaluate(field_out=field)
    plan = BlasmPlan(C, H, W, (pH, pW), cfg.wavelengths, cfg.distances(), cfg.pixel_pitch,
                     aperture_radius=cfg.resolved_aperture(), device=dev)
    levels = torch.empty((C, pH, pW), dtype=torch.uint8, device=dev)
    phase_field = torch.empty((C, pH, pW), dtype=torch.complex64, device=dev)
    _lib.check(_lib.lib().cvqpg_poh_encode(ctypes.byref(plan.params), _lib.ptr(plan.tables), plan.tables.numel(),
                                           _lib.ptr(torch.view_as_real(field)), _lib.ptr(levels),
                                           _lib.ptr(torch.view_as_real(phase_field)), _lib.stream_of(dev)),
               "cvqpg_poh_encode")
    ap = aperture_size if aperture_size is not None else min(W, H)
    recon = BlasmPlan(C, H, W, (pH, pW), cfg.wavelengths, cfg.distances(), cfg.pixel_pitch, aperture_radius=ap,
                      out_size=(H, W), input_mode=1, device=dev)
    V = recon.forward(phase_field)
    intensity = (V.real ** 2 + V.imag ** 2)
    img = intensity.clamp(0.0, 1.0)
    mse = ((img - fitter.targets) ** 2).mean(dim=(1, 2, 3)).double().cpu().numpy()
    return dict(levels=levels, phase_field=phase_field, intensity=intensity,
                psnr=-10.0 * np.log10(np.maximum(mse, 1e-30)), aperture=ap)
