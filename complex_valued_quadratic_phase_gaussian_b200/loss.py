"""Fused multi-plane loss + SSIM on the GPU, with dL/d(pred) from the same pass.

Mirror of the reference's loss for the fit loop:

* ``multiplane_loss_odak.__call__``  utils/propagator.py:417-449
  (L2 + masked L2 + correlation L2 against fresh target noise)
* ``GaussianLoss``                   utils/data_utils.py:22-41 (0.025 * 0.2 * (1 - SSIM))
* the per-plane loop                 train_2d_gaussian_rgb.py:192-199

``pred`` is the clamped intensity ``clamp(|V|^2, 0, 1)`` of every plane
([P, C, H, W] float32), which the BLASM inverse row pass writes. The noise is
Philox4x32-10 + Box-Muller keyed by (seed, iteration, element index), so the
same (seed, iteration) gives the same noisy target on every call.
"""
import ctypes

import torch

from . import _lib

TARGET_RANGE_WORKSPACE_PER_PLANE = 512  # CVQPG_TARGET_RANGE_WORKSPACE_PER_PLANE


class LossParams(ctypes.Structure):
    """``cvqpg_loss_params`` (include/cvqpg.h)."""
    _fields_ = [("channels", ctypes.c_int), ("planes", ctypes.c_int), ("height", ctypes.c_int),
                ("width", ctypes.c_int), ("w_l2", ctypes.c_float), ("w_mask", ctypes.c_float),
                ("w_cor", ctypes.c_float), ("ssim_weight", ctypes.c_float), ("noise_ratio", ctypes.c_float),
                ("inject_noise", ctypes.c_int), ("seed", ctypes.c_ulonglong), ("target_moments", ctypes.c_void_p)]


class MultiplaneLoss:
    """Loss of a fixed target stack; ``__call__`` returns (out, grad_pred).

    ``out`` is float32 [1 + 3P]: total loss, MSE of each plane, SSIM of each
    plane, loss of each plane. ``grad_pred`` is dL/d(pred), [P, C, H, W].
    """

    def __init__(self, targets, depth_plane, weights=(1.0, 1.0, 1.0), ssim_weight=0.025 * 0.2,
                 noise_ratio=1e-3, inject_noise=True, seed=0, target_moments=True):
        if targets.dim() != 4:
            raise ValueError("targets must be [planes, channels, height, width]")
        P, C, H, W = targets.shape
        self.targets = targets.contiguous().float()
        self.depth_plane = depth_plane.to(device=targets.device, dtype=torch.uint8).contiguous()
        if self.depth_plane.shape != (H, W):
            raise ValueError("depth_plane must be [height, width]")
        self.prm = LossParams(C, P, H, W, float(weights[0]), float(weights[1]), float(weights[2]),
                              float(ssim_weight), float(noise_ratio), int(bool(inject_noise)), int(seed))
        lib = _lib.lib()
        self.device = targets.device
        self.ws = _lib.workspace(_lib.size_query(lib.cvqpg_loss_workspace_size, ctypes.byref(self.prm)),
                                 self.device)
        self.target_range = torch.empty(P, dtype=torch.float32, device=self.device)
        _lib.check(lib.cvqpg_loss_target_range(_lib.ptr(self.targets), P, C, H, W, _lib.ptr(self.target_range),
                                               _lib.ptr(self.ws), self.ws.numel(), _lib.stream_of(self.device)),
                   "cvqpg_loss_target_range")
        self.moments = None
        if target_moments:  # the targets are fixed: filter them once (cvqpg_loss_target_moments)
            nbytes = _lib.size_query(lib.cvqpg_loss_target_moments_size, ctypes.byref(self.prm))
            self.moments = torch.empty(nbytes // 4, dtype=torch.float32, device=self.device)
            _lib.check(lib.cvqpg_loss_target_moments(ctypes.byref(self.prm), _lib.ptr(self.targets),
                                                     _lib.ptr(self.moments), nbytes, _lib.stream_of(self.device)),
                       "cvqpg_loss_target_moments")
            self.prm.target_moments = _lib.ptr(self.moments)
        self.shape = (P, C, H, W)

    def __call__(self, pred, iteration=0, out=None, grad_pred=None):
        if tuple(pred.shape) != self.shape or pred.dtype != torch.float32 or not pred.is_contiguous():
            raise ValueError(f"pred must be contiguous float32 {self.shape}")
        P = self.shape[0]
        if out is None:
            out = torch.empty(1 + 3 * P, dtype=torch.float32, device=self.device)
        if grad_pred is None:
            grad_pred = torch.empty_like(pred)
        if isinstance(iteration, torch.Tensor):
            it = iteration
        else:
            it = torch.tensor([int(iteration)], dtype=torch.int32, device=self.device)
        lib = _lib.lib()
        _lib.check(lib.cvqpg_loss_forward_backward(ctypes.byref(self.prm), _lib.ptr(pred), _lib.ptr(self.targets),
                                                   _lib.ptr(self.depth_plane), _lib.ptr(self.target_range),
                                                   _lib.ptr(it), _lib.ptr(grad_pred), _lib.ptr(out),
                                                   _lib.ptr(self.ws), self.ws.numel(), _lib.stream_of(self.device)),
                   "cvqpg_loss_forward_backward")
        return out, grad_pred
