"""Oracle: guard-band padding, amplitude clamp and BLASM propagation (numpy float64).

Test infrastructure only (see oracle/__init__.py). Restates, in the reference's
operation order,

* soft_window_pad                model_2d_gaussian_rgb.py:186-241
* phase/amplitude re-synthesis   train_2d_gaussian_rgb.py:89-95
  (angle(U) mod 2pi, clamp(|U|, 0, 1), amplitude * exp(i phase))
* propagator._reconstruct_impl   utils/propagator.py:248-290 with custom()
  (utils/propagator.py:41-64): zero_pad x2 -> fft2 -> fftshift -> x aperture
  -> x transfer function -> ifftshift -> ifft2 -> crop_center -> |.|^2
* the training crop              train_2d_gaussian_rgb.py:193
* the circular aperture          utils/propagator.py:10-38, 179-200

and the exact adjoints of the linear parts. The transfer function is the
odak restatement in oracle/odak_restated.py (parity unpinned).
"""
import numpy as np

from . import odak_restated as odr


def taper_1d(total, inner_start, inner_size):
    w = np.zeros(total)
    w[inner_start:inner_start + inner_size] = 1.0
    if inner_start > 0:
        t = np.arange(inner_start, dtype=np.float64)
        w[:inner_start] = 0.5 * (1.0 - np.cos(np.pi * (t + 1.0) / inner_start))
    right = inner_start + inner_size
    n_right = total - right
    if n_right > 0:
        t = np.arange(n_right, dtype=np.float64)
        w[right:] = 0.5 * (1.0 + np.cos(np.pi * (t + 1.0) / n_right))
    return w


def soft_window_pad(field, pH, pW):
    """[C,H,W] -> [C,pH,pW]: replicate guard band times a separable Tukey window."""
    field = np.asarray(field)
    C, H, W = field.shape
    ph, pw = (pH - H) // 2, (pW - W) // 2
    rows = np.clip(np.arange(pH) - ph, 0, H - 1)
    cols = np.clip(np.arange(pW) - pw, 0, W - 1)
    rep = field[:, rows][:, :, cols]
    win = np.outer(taper_1d(pH, ph, H), taper_1d(pW, pw, W))
    return rep * win[None]


def clamp_amplitude(u):
    a = np.abs(u)
    return np.where(a > 1.0, u / np.where(a > 0, a, 1.0), u)


def clamp_amplitude_adjoint(u, g):
    """Adjoint of clamp_amplitude under torch's angle/abs/clamp autograd conventions."""
    a = np.abs(u)
    r2 = a * a
    safe = np.where(r2 > 0, r2, 1.0)
    c, s = u.real / np.where(a > 0, a, 1.0), u.imag / np.where(a > 0, a, 1.0)
    gphi = -g.real * s + g.imag * c
    outer = (-gphi * u.imag / safe) + 1j * (gphi * u.real / safe)
    return np.where(r2 == 0, 0.0, np.where(r2 <= 1.0, g, outer))


def aperture_mask(NH, NW, radius):
    if radius is None or radius <= 0:
        return np.ones((NH, NW))
    x = np.linspace(-NH / 2.0, NH / 2.0, NH)
    y = np.linspace(-NW / 2.0, NW / 2.0, NW)
    X, Y = np.meshgrid(x, y, indexing="ij")
    return (np.sqrt(X ** 2 + Y ** 2) < radius).astype(np.float64)


def multiplier(NH, NW, dx, wavelength, distance, radius):
    """M such that the reference custom() equals ifft2(M * fft2(zero_pad(f)))."""
    Hc = odr.blasm_transfer_function(NH, NW, dx, wavelength, distance)
    A = aperture_mask(NH, NW, radius)
    return np.fft.ifftshift(Hc * A * A)


def _embed(x, NH, NW):
    C, h, w = x.shape
    out = np.zeros((C, NH, NW), dtype=np.complex128)
    r0, c0 = NH // 2 - h // 2, NW // 2 - w // 2
    out[:, r0:r0 + h, c0:c0 + w] = x
    return out


def _crop(z, h, w):
    NH, NW = z.shape[-2:]
    r0, c0 = NH // 2 - h // 2, NW // 2 - w // 2
    return z[..., r0:r0 + h, c0:c0 + w]


def propagate(x, wavelengths, distances, dx, out_hw, aperture_radius=None):
    """x [C,pH,pW] (already padded + clamped) -> V [P,C,oh,ow] complex128."""
    x = np.asarray(x, dtype=np.complex128)
    C, pH, pW = x.shape
    NH, NW = 2 * pH, 2 * pW
    oh, ow = out_hw
    F = np.fft.fft2(_embed(x, NH, NW))
    V = np.zeros((len(distances), C, oh, ow), dtype=np.complex128)
    for p, z in enumerate(distances):
        for c in range(C):
            M = multiplier(NH, NW, dx, wavelengths[c], float(z), aperture_radius)
            V[p, c] = _crop(np.fft.ifft2(M * F[c]), oh, ow)
    return V


def propagate_adjoint(gV, in_hw, wavelengths, distances, dx, aperture_radius=None):
    """Adjoint of propagate: gV [P,C,oh,ow] -> g [C,ih,iw] (ih, iw = pH, pW)."""
    gV = np.asarray(gV, dtype=np.complex128)
    P, C, oh, ow = gV.shape
    pH, pW = in_hw
    NH, NW = 2 * pH, 2 * pW
    acc = np.zeros((C, NH, NW), dtype=np.complex128)
    for p, z in enumerate(distances):
        G = np.fft.fft2(_embed(gV[p], NH, NW))
        for c in range(C):
            M = multiplier(NH, NW, dx, wavelengths[c], float(z), aperture_radius)
            acc[c] += np.conj(M) * G[c]
    return _crop(np.fft.ifft2(acc), pH, pW)


def chain_forward(field, pH, pW, wavelengths, distances, dx, out_hw=None, aperture_radius=None):
    """Splat field [C,H,W] -> pad/window -> clamp -> propagate -> V [P,C,oh,ow]."""
    C, H, W = field.shape
    U = soft_window_pad(field, pH, pW)
    return propagate(clamp_amplitude(U), wavelengths, distances, dx, out_hw or (H, W), aperture_radius)


def chain_backward(field, gV, pH, pW, wavelengths, distances, dx, aperture_radius=None):
    """dL/d(splat field) given dL/dV (the guard band carries no gradient)."""
    C, H, W = field.shape
    U = soft_window_pad(field, pH, pW)
    gx = propagate_adjoint(gV, (pH, pW), wavelengths, distances, dx, aperture_radius)
    gU = clamp_amplitude_adjoint(U, gx)
    ph, pw = (pH - H) // 2, (pW - W) // 2
    return gU[:, ph:ph + H, pw:pw + W]
