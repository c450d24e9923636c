"""Per-tile MLP of the learned initialiser on the sm_100a tensor cores.

The reference fits every hologram from a random Gaussian set; it has no
learned part. This module adds one: a small MLP maps each 16x16 tile of the
target (RGB + depth, 1024 values) to the raw parameters of 12 Gaussians
(12 x 13 = 156 values), trained on (target, converged fit) pairs produced by
the batched fitter. Its GEMMs are ``cvqpg_gemm_bf16_tn``: BF16 operands,
FP32 accumulation in tensor memory (tcgen05), fused bias / GELU / GELU'
epilogues.
"""
import ctypes

import torch

from . import _lib

EPI_F32, EPI_BIAS, EPI_BIAS_GELU, EPI_DGELU = 0, 1, 2, 3


class GemmEpilogue(ctypes.Structure):
    """``cvqpg_gemm_epilogue`` (include/cvqpg.h)."""
    _fields_ = [("mode", ctypes.c_int), ("valid_n", ctypes.c_int), ("bias", ctypes.c_void_p),
                ("zin", ctypes.c_void_p), ("ld_z", ctypes.c_int), ("ld_f32", ctypes.c_int),
                ("out_f32", ctypes.c_void_p), ("split_stride", ctypes.c_longlong), ("out_bf16", ctypes.c_void_p),
                ("out_bf16_t", ctypes.c_void_p), ("ld_bf16", ctypes.c_int), ("ld_t", ctypes.c_int)]


def _p(t):
    return None if t is None else _lib.ptr(t)


def gemm_bf16_tn(A, B, mode=EPI_F32, out_f32=None, bias=None, zin=None, out_bf16=None, out_bf16_t=None,
                 valid_n=0, splits=1, status=None):
    """C = A @ B.T on the tensor cores with a fused epilogue (see cvqpg_gemm_bf16_tn).

    A [M, K] and B [N, K] are BF16 CUDA tensors whose rows may be strided
    (``stride(1) == 1``). Outputs are written in place; returns ``status``
    (a device int32 tensor, non-zero if a pipeline wait timed out).
    """
    if A.dtype != torch.bfloat16 or B.dtype != torch.bfloat16 or A.stride(1) != 1 or B.stride(1) != 1:
        raise ValueError("A and B must be bfloat16 with contiguous rows")
    M, K = A.shape
    N = B.shape[0]
    if B.shape[1] != K:
        raise ValueError("A and B must share K")
    if status is None:
        status = torch.zeros(1, dtype=torch.int32, device=A.device)
    e = GemmEpilogue()
    e.mode = mode
    e.valid_n = int(valid_n)
    e.bias = _p(bias)
    e.zin = _p(zin)
    e.ld_z = zin.stride(0) if zin is not None else 0
    e.out_f32 = _p(out_f32)
    if out_f32 is not None:
        e.ld_f32 = out_f32.stride(-2)
        e.split_stride = out_f32.stride(0) if out_f32.dim() == 3 else 0
    e.out_bf16 = _p(out_bf16)
    e.ld_bf16 = out_bf16.stride(0) if out_bf16 is not None else 0
    e.out_bf16_t = _p(out_bf16_t)
    e.ld_t = out_bf16_t.stride(0) if out_bf16_t is not None else 0
    lib = _lib.lib()
    _lib.check(lib.cvqpg_gemm_bf16_tn(_lib.ptr(A), A.stride(0), _lib.ptr(B), B.stride(0), M, N, K, ctypes.byref(e),
                                      int(splits), _lib.ptr(status), _lib.stream_of(A.device)),
               "cvqpg_gemm_bf16_tn")
    return status
