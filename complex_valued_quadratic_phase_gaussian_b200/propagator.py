"""BLASM propagation on the B200 kernels, behind the reference propagator API.

* ``BlasmPlan`` owns the device tables for one geometry (hologram size, pad,
  wavelengths, plane distances, aperture) and runs the forward/adjoint kernels
  of libcvqpg.so (cvqpg_blasm_forward / cvqpg_blasm_backward).
* ``BlasmPropagate`` is the autograd Function: splat field [C,H,W] -> complex
  field at every plane [P,C,oh,ow] (intensity = |.|^2), fusing
  soft_window_pad (model_2d_gaussian_rgb.py:186-241), the amplitude clamp of
  reconstruct() (train_2d_gaussian_rgb.py:89-95), the propagation
  (utils/propagator.py:248-290) and the image crop (train_2d_gaussian_rgb.py:193).
* ``propagator`` mirrors the reference class (utils/propagator.py:67-290):
  same constructor arguments and ``reconstruct(hologram_phases, amplitude,
  no_grad)`` returning intensities [frames, planes, channels, pH, pW].
"""
import ctypes
import logging
import math

import torch
from torch.autograd import Function

from . import _lib


class BlasmParams(ctypes.Structure):
    _fields_ = [("channels", ctypes.c_int), ("planes", ctypes.c_int), ("height", ctypes.c_int),
                ("width", ctypes.c_int), ("pad_height", ctypes.c_int), ("pad_width", ctypes.c_int),
                ("out_height", ctypes.c_int), ("out_width", ctypes.c_int), ("input_mode", ctypes.c_int),
                ("plan_hint", ctypes.c_int), ("pixel_pitch", ctypes.c_double),
                ("wavelengths", ctypes.c_double * 3), ("distances", ctypes.c_double * 8),
                ("aperture_radius", ctypes.c_double)]


def reference_distances(num_planes, volume_depth, d_val):
    """Plane distances exactly as the training script builds them (float32 linspace + offset,
    train_2d_gaussian_rgb.py:360-363)."""
    if num_planes > 1:
        d = torch.linspace(-volume_depth / 2.0, volume_depth / 2.0, num_planes) + d_val
        return [float(v) for v in d.tolist()]
    return [float(d_val)]


def reference_pad_size(img_size):
    """Default guard band of the training script (train_2d_gaussian_rgb.py:340-343); img_size = (W, H)."""
    W, H = img_size
    return [((H + 2 * 144 + 63) // 64) * 64, ((W + 2 * 144 + 63) // 64) * 64]


class BlasmPlan:
    """Device tables + workspace for one propagation geometry."""

    def __init__(self, channels, height, width, pad_size, wavelengths, distances, pixel_pitch,
                 aperture_radius=None, out_size=None, input_mode=0, device="cuda", plan_hint=0):
        if len(distances) > 8:
            raise ValueError("at most 8 planes are supported")
        self.device = torch.device(device)
        p = BlasmParams()
        p.channels, p.planes = int(channels), len(distances)
        p.height, p.width = int(height), int(width)
        p.pad_height, p.pad_width = int(pad_size[0]), int(pad_size[1])
        oh, ow = out_size if out_size is not None else (height, width)
        p.out_height, p.out_width = int(oh), int(ow)
        p.input_mode = int(input_mode)
        p.pixel_pitch = float(pixel_pitch)
        for i, wl in enumerate(wavelengths):
            p.wavelengths[i] = float(wl)
        for i, z in enumerate(distances):
            p.distances[i] = float(z)
        p.aperture_radius = float(aperture_radius) if aperture_radius else 0.0
        p.plan_hint = int(plan_hint)
        self.params = p
        lib = _lib.lib()
        pp = ctypes.byref(p)
        nbytes = _lib.size_query(lib.cvqpg_blasm_tables_size, pp)
        with torch.cuda.device(self.device):
            self.tables = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            _lib.check(lib.cvqpg_blasm_setup(pp, _lib.ptr(self.tables), nbytes), "cvqpg_blasm_setup")
        self.ws_bytes = _lib.size_query(lib.cvqpg_blasm_workspace_size, pp)
        self._ws = None
        self.C, self.P = p.channels, p.planes
        self.in_shape = (p.channels, p.height, p.width) if input_mode == 0 else (p.channels, p.pad_height, p.pad_width)
        self.out_shape = (p.planes, p.channels, p.out_height, p.out_width)

    def workspace(self):
        if self._ws is None:
            self._ws = _lib.workspace(self.ws_bytes, self.device)
        return self._ws

    def forward(self, field, out=None):
        field = field.contiguous()
        if field.dtype != torch.complex64 or tuple(field.shape) != self.in_shape:
            raise RuntimeError(f"field must be complex64 {self.in_shape}, got {field.dtype} {tuple(field.shape)}")
        if out is None:
            out = torch.empty(self.out_shape, dtype=torch.complex64, device=self.device)
        ws = self.workspace()
        _lib.check(_lib.lib().cvqpg_blasm_forward(
            ctypes.byref(self.params), _lib.ptr(self.tables), self.tables.numel(),
            _lib.ptr(torch.view_as_real(field)), _lib.ptr(torch.view_as_real(out)), _lib.ptr(ws), ws.numel(),
            _lib.stream_of(self.device)), "cvqpg_blasm_forward")
        return out

    def backward(self, field, grad_out, out=None):
        grad_out = grad_out.resolve_conj().contiguous()
        if out is None:
            out = torch.empty(self.in_shape, dtype=torch.complex64, device=self.device)
        ws = self.workspace()
        fptr = _lib.ptr(torch.view_as_real(field.contiguous())) if field is not None else None
        _lib.check(_lib.lib().cvqpg_blasm_backward(
            ctypes.byref(self.params), _lib.ptr(self.tables), self.tables.numel(), fptr,
            _lib.ptr(torch.view_as_real(grad_out)), _lib.ptr(torch.view_as_real(out)), _lib.ptr(ws), ws.numel(),
            _lib.stream_of(self.device)), "cvqpg_blasm_backward")
        return out


class BlasmPropagate(Function):
    """field [C,H,W] (mode 0) or padded field [C,pH,pW] (mode 1) -> V [P,C,oh,ow]."""

    @staticmethod
    def forward(ctx, field, plan):
        field = field.contiguous()
        ctx.plan = plan
        ctx.save_for_backward(field)
        return plan.forward(field)

    @staticmethod
    def backward(ctx, grad_v):
        (field,) = ctx.saved_tensors
        return ctx.plan.backward(field, grad_v), None


def blasm_propagate(field, plan):
    return BlasmPropagate.apply(field, plan)


class propagator:
    """Reference-compatible propagator (utils/propagator.py:67-290) running on libcvqpg.

    ``reconstruct(hologram_phases, amplitude=None, no_grad=True)`` returns
    intensities [number_of_frames, depth_layers, channels, pH, pW] exactly like
    the reference (frames whose laser power is zero for a channel are skipped,
    utils/propagator.py:280-283).
    """

    def __init__(self, resolution=(1920, 1080), wavelengths=(515e-9,), pixel_pitch=8e-6, number_of_frames=1,
                 number_of_depth_layers=1, volume_depth=1e-2, image_location_offset=5e-3,
                 propagation_type="Bandlimited Angular Spectrum", laser_channel_power=None, aperture=None,
                 aperture_size=None, distances=None, aperture_samples=(20, 20, 5, 5), device=torch.device("cuda")):
        if propagation_type != "Bandlimited Angular Spectrum":
            raise ValueError("only 'Bandlimited Angular Spectrum' propagation is implemented")
        if aperture is not None:
            raise ValueError("a custom aperture tensor is not supported; use aperture_size")
        self.device = torch.device(device)
        self.resolution = list(resolution)
        self.wavelengths = list(wavelengths)
        self.pixel_pitch = pixel_pitch
        self.number_of_frames = number_of_frames
        self.number_of_channels = len(self.wavelengths)
        if distances is None:
            d = torch.linspace(-volume_depth / 2.0, volume_depth / 2.0, number_of_depth_layers) + image_location_offset
        else:
            d = torch.as_tensor(distances)
        self.distances = d
        self.number_of_depth_layers = int(d.shape[0])
        if laser_channel_power is None:
            laser_channel_power = torch.eye(number_of_frames, self.number_of_channels)
        self.channel_power = laser_channel_power.to(self.device)
        self._power = laser_channel_power.detach().cpu().float()
        if aperture_size is None:
            aperture_size = max(self.resolution[0], self.resolution[1])
        self.aperture_size = aperture_size
        pH, pW = self.resolution
        self.plan = BlasmPlan(self.number_of_channels, pH, pW, (pH, pW), self.wavelengths,
                              [float(z) for z in d.tolist()], pixel_pitch, aperture_radius=aperture_size,
                              out_size=(pH, pW), input_mode=1, device=self.device)

    def reconstruct(self, hologram_phases, amplitude=None, no_grad=True):
        if no_grad:
            with torch.no_grad():
                return self._reconstruct_impl(hologram_phases, amplitude)
        return self._reconstruct_impl(hologram_phases, amplitude)

    def _reconstruct_impl(self, hologram_phases, amplitude=None):
        if hologram_phases.dim() > 3:
            hologram_phases = hologram_phases.squeeze(0)
        if hologram_phases.shape[0] != self.number_of_frames:
            logging.warning("Provided hologram frame count is %d but the configured number of frames is %d.",
                            hologram_phases.shape[0], self.number_of_frames)
        C = self.number_of_channels
        pH, pW = self.resolution
        if amplitude is None:
            amplitude = torch.ones(C, pH, pW, device=self.device)
        frames = []
        for f in range(self.number_of_frames):
            power = self._power[f]
            phase = hologram_phases[f]
            x = torch.stack([torch.polar((float(power[c]) * amplitude[c]).float(), phase.float()) for c in range(C)])
            I = blasm_propagate(x.to(torch.complex64), self.plan).abs().pow(2)  # [P, C, pH, pW]
            mask = torch.tensor([float(power[c] != 0) for c in range(C)], device=I.device).view(1, C, 1, 1)
            frames.append(I * mask)
        return torch.stack(frames)
