"""Drop-in replacement for the reference ``cuda/rasterizer.py`` (QPF rasterizer).

Same public names and argument meaning as the reference module:

* ``qpf_render(means_2d, inv_cov, colours, phase, opacities, curvature, area,
  radii, k, dxy2, width, height) -> complex64 [C, H, W]``
  (reference cuda/rasterizer.py:62-71)
* ``QPFRender`` autograd Function (reference cuda/rasterizer.py:36-59)
* ``ext()`` returning an object with ``qpf_render_forward`` /
  ``qpf_render_backward`` that take and return the same tensors as the
  reference pybind module (cuda/binding.cpp:4-7, cuda/raster.cu:30-143).

The work is done by libcvqpg.so (sm_100a) through its C ABI; there is no CPU
path. Errors are raised as RuntimeError with the reference's TORCH_CHECK texts
(cuda/raster.cu:22-28, 45; cuda/forward.cu:173).
"""
import torch
from torch.autograd import Function

from . import _lib

CULL_CUDA16_5SIGMA = 0
CULL_TORCH64_3SIGMA = 1
CULL_NONE = 2
PHASE_ISO = 0x100  # OR-ed into the cull mode: isotropic quadratic phase (reference --phase_iso)

_capacity_hint = {}


def _check_input(t, name, n):
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be CUDA")
    if not t.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")
    if t.dtype not in (torch.float32, torch.int32):
        raise RuntimeError(f"{name} must be float32/int32")
    if t.size(0) != n:
        raise RuntimeError(f"{name} has {t.size(0)} rows, expected {n}")


def _check_channels(c):
    if c not in (1, 3):
        raise RuntimeError(f"qpf rasterizer supports 1 or 3 channels, got {c}")


def render_forward(means_2d, inv_cov, colours, phase, opacities, curvature, area, k, dxy2, width, height,
                   cull=CULL_CUDA16_5SIGMA, radii=None, radius3=None, phase_iso=False):
    """Run binning + splat. Returns (field complex64 [C,H,W], point_list, ranges).

    phase_iso: isotropic quadratic phase 0.5 c |r - mu|^2 dxy2 (the torch renderer's
    --phase_iso) instead of the Mahalanobis form 0.5 c m area dxy2.

    ``point_list`` holds exactly the produced pairs (the reference's
    ``total_pairs``; a single zero when there are none, cuda/raster.cu:72-75).
    """
    n = means_2d.size(0)
    c = colours.size(1) if colours.dim() == 2 else 1
    _check_channels(c)
    named = [(means_2d, "means_2d"), (inv_cov, "inv_cov"), (colours, "colours"), (phase, "phase"),
             (opacities, "opacities"), (curvature, "curvature"), (area, "area")]
    if cull == CULL_CUDA16_5SIGMA:
        named.append((radii, "radii"))
    elif cull == CULL_TORCH64_3SIGMA:
        named.append((radius3, "radius3"))
    for t, name in named:
        _check_input(t, name, n)
    if k.numel() != c:
        raise RuntimeError("k must have num_channels entries")
    dev = means_2d.device
    lib = _lib.lib()
    with torch.cuda.device(dev):
        num_lists = lib.cvqpg_render_num_lists(cull, int(width), int(height))
        out = torch.empty((c, int(height), int(width)), dtype=torch.complex64, device=dev)
        ranges = torch.empty((num_lists, 2), dtype=torch.int32, device=dev)
        pair_count = torch.zeros(2, dtype=torch.int32, device=dev)
        key = (n, int(width), int(height), cull)
        cap = _capacity_hint.get(key, max(1024, 8 * n))
        while True:
            ws = _lib.workspace(_lib.size_query(lib.cvqpg_render_workspace_size, n, int(width), int(height), cap),
                                dev)
            point_list = torch.empty(max(cap, 1), dtype=torch.int32, device=dev)
            _lib.check(lib.cvqpg_render_forward_cull(
                _lib.ptr(means_2d), _lib.ptr(inv_cov), _lib.ptr(colours), _lib.ptr(phase), _lib.ptr(opacities),
                _lib.ptr(curvature), _lib.ptr(area), int(cull) | (PHASE_ISO if phase_iso else 0), _lib.ptr(radii),
                _lib.ptr(radius3),
                _lib.ptr(k), float(dxy2), n, int(width), int(height), c, _lib.ptr(torch.view_as_real(out)),
                _lib.ptr(point_list), cap, _lib.ptr(ranges), _lib.ptr(pair_count), _lib.ptr(ws), ws.numel(),
                _lib.stream_of(dev)), "qpf_render_forward")
            total, over = (int(v) for v in pair_count.tolist())  # host sync, as cuda/raster.cu:71
            if not over:
                break
            cap = int(total * 1.25) + 1024
        _capacity_hint[key] = max(cap, int(total * 1.25) + 1024)
    if total <= 0:
        point_list = torch.zeros(1, dtype=torch.int32, device=dev)
    else:
        point_list = point_list[:total]
    return out, point_list, ranges


def render_backward(grad_field, means_2d, inv_cov, colours, phase, opacities, curvature, area, k, point_list,
                    ranges, dxy2, width, height, cull=CULL_CUDA16_5SIGMA, phase_iso=False):
    """Adjoint of render_forward; returns the 7 input gradients."""
    n = means_2d.size(0)
    c = colours.size(1) if colours.dim() == 2 else 1
    _check_channels(c)
    dev = means_2d.device
    lib = _lib.lib()
    g = grad_field.resolve_conj().contiguous()
    if g.dtype != torch.complex64:
        g = g.to(torch.complex64)
    with torch.cuda.device(dev):
        d_means = torch.empty((n, 2), dtype=torch.float32, device=dev)
        d_inv = torch.empty((n, 3), dtype=torch.float32, device=dev)
        d_col = torch.empty((n, c), dtype=torch.float32, device=dev)
        d_ph = torch.empty((n, c), dtype=torch.float32, device=dev)
        d_op = torch.empty((n,), dtype=torch.float32, device=dev)
        d_cv = torch.empty((n,), dtype=torch.float32, device=dev)
        d_ar = torch.empty((n,), dtype=torch.float32, device=dev)
        ws = _lib.workspace(_lib.size_query(lib.cvqpg_render_backward_workspace_size, n), dev)
        _lib.check(lib.cvqpg_render_backward_cull(
            _lib.ptr(torch.view_as_real(g)), _lib.ptr(means_2d), _lib.ptr(inv_cov), _lib.ptr(colours),
            _lib.ptr(phase), _lib.ptr(opacities), _lib.ptr(curvature), _lib.ptr(area), _lib.ptr(k),
            int(cull) | (PHASE_ISO if phase_iso else 0),
            _lib.ptr(point_list), _lib.ptr(ranges), float(dxy2), n, int(width), int(height), c,
            _lib.ptr(d_means), _lib.ptr(d_inv), _lib.ptr(d_col), _lib.ptr(d_ph), _lib.ptr(d_op), _lib.ptr(d_cv),
            _lib.ptr(d_ar), _lib.ptr(ws), ws.numel(), _lib.stream_of(dev)), "qpf_render_backward")
    return [d_means, d_inv, d_col, d_ph, d_op, d_cv, d_ar]


class _Ext:
    """Tensor-level mirror of the reference pybind module ``qpf_2d_cuda``."""

    @staticmethod
    def qpf_render_forward(means_2d, inv_cov, colours, phase, opacities, curvature, area, radii, k, dxy2,
                           width, height, num_channels):
        if colours.size(1) != num_channels:
            raise RuntimeError("colours must have num_channels columns")
        _check_channels(num_channels)
        if k.numel() != num_channels:
            raise RuntimeError("k must have num_channels entries")
        out, point_list, ranges = render_forward(means_2d, inv_cov, colours, phase, opacities, curvature, area, k,
                                                 dxy2, width, height, CULL_CUDA16_5SIGMA, radii=radii)
        return [out.real.contiguous(), out.imag.contiguous(), point_list, ranges]

    @staticmethod
    def qpf_render_backward(grad_real, grad_imag, means_2d, inv_cov, colours, phase, opacities, curvature, area,
                            k, point_list, ranges, dxy2, width, height, num_channels):
        _check_channels(num_channels)
        g = torch.complex(grad_real.contiguous(), grad_imag.contiguous())
        return render_backward(g, means_2d, inv_cov, colours, phase, opacities, curvature, area, k, point_list,
                               ranges, dxy2, width, height, CULL_CUDA16_5SIGMA)


_EXT = _Ext()


def ext():
    """Return the kernel module (the reference compiles it here on first use)."""
    _lib.lib()
    return _EXT


class QPFRender(Function):
    """Autograd wrapper, same inputs/gradients as reference cuda/rasterizer.py:36-59."""

    @staticmethod
    def forward(ctx, means_2d, inv_cov, colours, phase, opacities, curvature, area, radii, k, dxy2, width, height):
        args = [t.contiguous() for t in (means_2d, inv_cov, colours, phase, opacities, curvature, area)]
        kk = k.contiguous()
        out, point_list, ranges = render_forward(*args, kk, dxy2, width, height, CULL_CUDA16_5SIGMA,
                                                 radii=radii.contiguous().int())
        ctx.save_for_backward(*args, kk, point_list, ranges)
        ctx.cfg = (float(dxy2), int(width), int(height))
        return out

    @staticmethod
    def backward(ctx, grad_out):
        (means, inv_cov, colours, phase, opac, curv, area, k, point_list, ranges) = ctx.saved_tensors
        dxy2, w, h = ctx.cfg
        d = render_backward(grad_out, means, inv_cov, colours, phase, opac, curv, area, k, point_list, ranges,
                            dxy2, w, h, CULL_CUDA16_5SIGMA)
        return d[0], d[1], d[2], d[3], d[4], d[5], d[6], None, None, None, None, None


class QPFRenderCull(Function):
    """QPFRender with an explicit culling rule (CULL_* constants of this module)."""

    @staticmethod
    def forward(ctx, means_2d, inv_cov, colours, phase, opacities, curvature, area, k, dxy2, width, height, cull,
                radii, radius3, phase_iso=False):
        args = [t.contiguous() for t in (means_2d, inv_cov, colours, phase, opacities, curvature, area)]
        kk = k.contiguous()
        out, point_list, ranges = render_forward(
            *args, kk, dxy2, width, height, cull,
            radii=None if radii is None else radii.contiguous().int(),
            radius3=None if radius3 is None else radius3.detach().contiguous().float(), phase_iso=phase_iso)
        ctx.save_for_backward(*args, kk, point_list, ranges)
        ctx.cfg = (float(dxy2), int(width), int(height), int(cull), bool(phase_iso))
        return out

    @staticmethod
    def backward(ctx, grad_out):
        (means, inv_cov, colours, phase, opac, curv, area, k, point_list, ranges) = ctx.saved_tensors
        dxy2, w, h, cull, iso = ctx.cfg
        d = render_backward(grad_out, means, inv_cov, colours, phase, opac, curv, area, k, point_list, ranges,
                            dxy2, w, h, cull, phase_iso=iso)
        return (d[0], d[1], d[2], d[3], d[4], d[5], d[6]) + (None,) * 8


def qpf_render(means_2d, inv_cov, colours, phase, opacities, curvature, area, radii, k, dxy2, width, height):
    """Complex field [C, H, W] of N Gaussians (linear coherent sum, quadratic phase).

    means_2d [N,2] pixel coords, inv_cov [N,3] = (inv00, inv01, inv11), colours/phase [N,C],
    opacities/curvature/area [N] (area = |sx*sy|), radii [N] culling radius in px,
    k [C] wavenumbers, dxy2 = pixel_pitch**2.
    """
    return QPFRender.apply(means_2d, inv_cov, colours, phase, opacities, curvature, area, radii, k, dxy2, width,
                           height)


def qpf_render_cull(means_2d, inv_cov, colours, phase, opacities, curvature, area, k, dxy2, width, height,
                    cull=CULL_CUDA16_5SIGMA, radii=None, radius3=None, phase_iso=False):
    """qpf_render with an explicit culling rule (for like-with-like parity checks) and optionally the
    isotropic quadratic phase of the torch renderer's --phase_iso (model_2d_gaussian_rgb.py:356-359)."""
    return QPFRenderCull.apply(means_2d, inv_cov, colours, phase, opacities, curvature, area, k, dxy2, width,
                               height, cull, radii, radius3, phase_iso)
