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


class MlpParams(ctypes.Structure):
    """``cvqpg_mlp_params`` (include/cvqpg.h)."""
    _fields_ = [("batch", ctypes.c_int), ("in_dim", ctypes.c_int), ("hidden", ctypes.c_int), ("out_dim", ctypes.c_int),
                ("lr", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float), ("eps", ctypes.c_float),
                ("weight_decay", ctypes.c_float), ("reserved", ctypes.c_int)]


class TileMLP:
    """in_dim -> hidden -> hidden -> out_dim MLP with GELU, trained with Adam on the GPU.

    ``weights`` is the flat FP32 vector of cvqpg.h (W1 | b1 | W2 | b2 | W3 | b3,
    W3/b3 padded to a multiple of 128 rows). One instance serves one batch size.
    """

    def __init__(self, batch, in_dim=1024, hidden=512, out_dim=156, lr=3e-4, betas=(0.9, 0.999), eps=1e-8,
                 weight_decay=0.0, weights=None, device="cuda"):
        self.device = torch.device(device)
        self.prm = MlpParams(int(batch), int(in_dim), int(hidden), int(out_dim), float(lr), float(betas[0]),
                             float(betas[1]), float(eps), float(weight_decay), 0)
        lib = _lib.lib()
        n = _lib.size_query(lib.cvqpg_mlp_weights_size, ctypes.byref(self.prm))
        self.ws = _lib.workspace(_lib.size_query(lib.cvqpg_mlp_workspace_size, ctypes.byref(self.prm)), self.device)
        if weights is None:
            from_numpy = _default_init(in_dim, hidden, out_dim)
            weights = torch.from_numpy(from_numpy)
        self.weights = torch.as_tensor(weights, dtype=torch.float32).to(self.device).contiguous()
        if self.weights.numel() != n:
            raise ValueError(f"weights must have {n} floats")
        self.adam = torch.zeros(2 * n, dtype=torch.float32, device=self.device)
        self.step_count = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        self.sync()

    def sync(self):
        """Refresh the BF16 weight copies after writing ``weights`` from outside."""
        lib = _lib.lib()
        _lib.check(lib.cvqpg_mlp_sync_weights(ctypes.byref(self.prm), _lib.ptr(self.weights), _lib.ptr(self.ws),
                                              self.ws.numel(), _lib.stream_of(self.device)), "cvqpg_mlp_sync_weights")

    def forward(self, X, out=None):
        X = X.contiguous().float()
        if out is None:
            out = torch.empty((self.prm.batch, self.prm.out_dim), dtype=torch.float32, device=self.device)
        lib = _lib.lib()
        _lib.check(lib.cvqpg_mlp_forward(ctypes.byref(self.prm), _lib.ptr(self.weights), _lib.ptr(X), _lib.ptr(out),
                                         _lib.ptr(self.ws), self.ws.numel(), _lib.ptr(self.status),
                                         _lib.stream_of(self.device)), "cvqpg_mlp_forward")
        return out

    def gradients(self, X, T, out_weight):
        grads = torch.empty_like(self.weights)
        lib = _lib.lib()
        _lib.check(lib.cvqpg_mlp_gradients(ctypes.byref(self.prm), _lib.ptr(self.weights), _lib.ptr(X.contiguous()),
                                           _lib.ptr(T.contiguous()), _lib.ptr(out_weight.contiguous()),
                                           _lib.ptr(grads), _lib.ptr(self.loss), _lib.ptr(self.ws), self.ws.numel(),
                                           _lib.ptr(self.status), _lib.stream_of(self.device)), "cvqpg_mlp_gradients")
        return self.loss, grads

    def adam_step(self, grads):
        """One Adam step from given gradients (e.g. after a data-parallel all-reduce)."""
        lib = _lib.lib()
        _lib.check(lib.cvqpg_mlp_adam_step(ctypes.byref(self.prm), _lib.ptr(self.weights), _lib.ptr(self.adam),
                                           _lib.ptr(self.step_count), _lib.ptr(grads.contiguous()), _lib.ptr(self.ws),
                                           self.ws.numel(), _lib.stream_of(self.device)), "cvqpg_mlp_adam_step")

    def data_parallel_step(self, X, T, out_weight, group=None):
        """One data-parallel step: this rank's shard (X, T) -> gradients on the tensor cores ->
        all-reduce weighted by rows -> the same Adam step on every rank. Returns the global loss."""
        loss, grads = data_parallel_gradients(lambda: self.gradients(X, T, out_weight), X.shape[0], group)
        self.adam_step(grads)
        return loss

    def train_step(self, X, T, out_weight):
        """One Adam step on (X, T); returns the device loss tensor (no host sync)."""
        lib = _lib.lib()
        _lib.check(lib.cvqpg_mlp_train_step(ctypes.byref(self.prm), _lib.ptr(self.weights), _lib.ptr(self.adam),
                                            _lib.ptr(self.step_count), _lib.ptr(X), _lib.ptr(T), _lib.ptr(out_weight),
                                            _lib.ptr(self.loss), _lib.ptr(self.ws), self.ws.numel(),
                                            _lib.ptr(self.status), _lib.stream_of(self.device)),
                   "cvqpg_mlp_train_step")
        return self.loss


def data_parallel_gradients(grad_fn, rows, group=None):
    """Average per-rank gradients into the full-batch gradient of the mean loss.

    grad_fn() returns (loss, grads) of this rank's shard of `rows` rows (mean over its rows).
    The shards may differ in size: each rank's gradient and loss are weighted by its row
    count in one all-reduce of [grads | loss | rows] (NCCL on GPUs, gloo on CPUs)."""
    import torch.distributed as dist
    loss, grads = grad_fn()
    buf = torch.cat([grads.reshape(-1) * rows, torch.as_tensor(loss, dtype=grads.dtype, device=grads.device)
                     .reshape(1) * rows, torch.tensor([float(rows)], dtype=grads.dtype, device=grads.device)])
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(buf, group=group)
    total = buf[-1]
    return buf[-2] / total, (buf[:-2] / total).reshape(grads.shape)


def _default_init(in_dim, hidden, out_dim, seed=0):
    """He-normal hidden layers, a small output layer, zero biases (float32, flat layout)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    op = (out_dim + 127) // 128 * 128
    w1 = rng.normal(0, np.sqrt(2.0 / in_dim), (hidden, in_dim))
    w2 = rng.normal(0, np.sqrt(2.0 / hidden), (hidden, hidden))
    w3 = np.zeros((op, hidden))
    w3[:out_dim] = rng.normal(0, 0.1 / np.sqrt(hidden), (out_dim, hidden))
    return np.concatenate([w1.ravel(), np.zeros(hidden), w2.ravel(), np.zeros(hidden), w3.ravel(),
                           np.zeros(op)]).astype(np.float32)
