"""Restatement of the odak 0.2.7 functions the reference calls -- TEST INFRASTRUCTURE ONLY.

odak (requirements.txt:4, pinned 0.2.7) is not installed on this machine and
cannot be fetched, so these functions are written from the published
mathematics, not from odak's code. Parity for them is UNPINNED; the reference
call sites they stand in for are:

  utils/propagator.py:6-7, 60, 210-220, 284-289, 407
  train_2d_gaussian_rgb.py:92-93, 103, 193

Conventions assumed (stated so that a later run against the real package can
confirm or correct them):

* ``zero_pad`` centres the field: start index = N//2 - n//2 on each of the last
  two axes; default target size = 2x.
* ``crop_center`` is its inverse: default keeps the centre half starting at
  N//4; with ``size`` keeps [N//2 - s//2, N//2 + s//2).
* ``get_propagation_kernel(..., 'Bandlimited Angular Spectrum')`` is the
  band-limited angular spectrum transfer function of K. Matsushima and
  T. Shimobaba, "Band-limited angular spectrum method for numerical simulation
  of free-space propagation in far and near fields", Opt. Express 17(22),
  19662 (2009):
      H(fx, fy) = exp(i 2 pi z sqrt(1/lambda^2 - fx^2 - fy^2))
                  * [|fx| < f_lim,x] * [|fy| < f_lim,y],
      f_lim,x = 1 / (lambda sqrt((2 z / S_x)^2 + 1)),  S_x = nu * dx,
  sampled on the symmetric grid fx_j = -1/(2 dx) + 1/(4 S_x) + j * step,
  j = 0..nu-1, step = (1/dx - 1/(2 S_x)) / (nu - 1) (same for y with nv).
  It is evaluated in float64 and rounded once to complex64, i.e. without the
  float32 evaluation error (~1e-3 rad at these distances) of a float32 graph.
* ``generate_2d_gaussian`` samples 1/(2 pi sx sy) exp(-(x^2/2sx^2 + y^2/2sy^2))
  on linspace(-L/2, L/2, L) per axis, with a zero sigma replaced by 1e-5
  (so the in-focus kernel is a unit impulse after normalisation).
"""
import math

import numpy as np
import torch


def zero_pad(field, size=None, method="center"):
    orig_dim = field.dim()
    f = field
    while f.dim() < 4:
        f = f.unsqueeze(0)
    n0, n1 = f.shape[-2], f.shape[-1]
    if size is None:
        N0, N1 = 2 * n0, 2 * n1
    else:
        N0, N1 = int(size[0]), int(size[1])
    out = torch.zeros(f.shape[:-2] + (N0, N1), dtype=f.dtype, device=f.device)
    s0, s1 = N0 // 2 - n0 // 2, N1 // 2 - n1 // 2
    out[..., s0:s0 + n0, s1:s1 + n1] = f
    while out.dim() > orig_dim:
        out = out.squeeze(0)
    return out


def crop_center(field, size=None):
    if size is None:
        N0, N1 = field.shape[-2], field.shape[-1]
        q0, q1 = N0 // 4, N1 // 4
        return field[..., q0:q0 + N0 // 2, q1:q1 + N1 // 2]
    c0, c1 = field.shape[-2] // 2, field.shape[-1] // 2
    h0, h1 = int(size[0]) // 2, int(size[1]) // 2
    return field[..., c0 - h0:c0 + h0, c1 - h1:c1 + h1]


def generate_complex_field(amplitude, phase):
    if not torch.is_tensor(amplitude):
        amplitude = torch.tensor(amplitude)
    return amplitude * torch.cos(phase) + 1j * amplitude * torch.sin(phase)


def calculate_amplitude(field):
    return torch.abs(field)


def calculate_phase(field):
    return torch.angle(field)


def blasm_frequency_grid(n, dx):
    """Symmetric frequency samples of one axis (float64)."""
    s = dx * float(n)
    return np.linspace(-1.0 / (2.0 * dx) + 0.5 / (2.0 * s), 1.0 / (2.0 * dx) - 0.5 / (2.0 * s), n)


def blasm_band_limit(n, dx, wavelength, distance):
    s = dx * float(n)
    return 1.0 / math.sqrt((2.0 * distance * (1.0 / s)) ** 2 + 1.0) / wavelength


def blasm_transfer_function(nu, nv, dx, wavelength, distance):
    """H on the nu x nv grid, complex128 (rows follow fx, columns fy)."""
    fx = blasm_frequency_grid(nu, dx)
    fy = blasm_frequency_grid(nv, dx)
    FX, FY = np.meshgrid(fx, fy, indexing="ij")
    arg = 1.0 / wavelength ** 2 - (FX ** 2 + FY ** 2)
    keep = (np.abs(FX) < blasm_band_limit(nu, dx, wavelength, distance)) & \
           (np.abs(FY) < blasm_band_limit(nv, dx, wavelength, distance)) & (arg >= 0)
    ph = 2.0 * np.pi * np.sqrt(np.maximum(arg, 0.0)) * distance
    return np.where(keep, np.exp(1j * ph), 0.0)


def get_propagation_kernel(nu, nv, dx=8e-6, wavelength=515e-9, distance=0.0, device=torch.device("cpu"),
                           propagation_type="Bandlimited Angular Spectrum", samples=(20, 20, 5, 5), scale=1):
    if propagation_type != "Bandlimited Angular Spectrum":
        raise NotImplementedError(propagation_type)
    if torch.is_tensor(distance):
        distance = float(distance.item())
    H = blasm_transfer_function(int(nu), int(nv), float(dx), float(wavelength), float(distance))
    return torch.from_numpy(H.astype(np.complex64)).to(device)


def generate_2d_gaussian(kernel_length=(21, 21), nsigma=(3, 3), mu=(0, 0), normalize=False):
    L0, L1 = int(kernel_length[0]), int(kernel_length[1])
    s0 = float(nsigma[0]) if float(nsigma[0]) != 0 else 1e-5
    s1 = float(nsigma[1]) if float(nsigma[1]) != 0 else 1e-5
    x = torch.linspace(-L0 / 2.0, L0 / 2.0, L0)
    y = torch.linspace(-L1 / 2.0, L1 / 2.0, L1)
    X, Y = torch.meshgrid(x, y, indexing="ij")
    k = 1.0 / (2.0 * math.pi * s0 * s1) * torch.exp(
        -((X - mu[0]) ** 2 / (2.0 * s0 ** 2) + (Y - mu[1]) ** 2 / (2.0 * s1 ** 2)))
    if normalize:
        k = k / k.max()
    return k
