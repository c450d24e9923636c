"""ctypes binding of ``libcvqpg.so`` (the C ABI declared in include/cvqpg.h).

The library is loaded from this package directory. There is no fallback: if
the library is missing or a call fails, a RuntimeError is raised. Tensors cross
the boundary as raw device pointers; streams as the current torch stream handle.
"""
import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcvqpg.so")

_p = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float
_d = ctypes.c_double
_sz = ctypes.c_size_t
_u64 = ctypes.c_uint64
_psz = ctypes.POINTER(ctypes.c_size_t)

# name -> argument types (all return int status unless listed in _RESTYPES)
_SIGNATURES = {
    "cvqpg_status_string": [_i],
    "cvqpg_version": [],
    "cvqpg_render_workspace_size": [_i, _i, _i, _i, _psz],
    "cvqpg_render_num_lists": [_i, _i, _i],
    "cvqpg_render_forward": [_p, _p, _p, _p, _p, _p, _p, _p, _p, _f, _i, _i, _i, _i,
                             _p, _p, _i, _p, _p, _p, _sz, _p],
    "cvqpg_render_forward_noalloc": [_p, _p, _p, _p, _p, _p, _p, _p, _p, _f, _i, _i, _i, _i,
                                     _p, _p, _i, _p, _p, _p],
    "cvqpg_render_forward_cull": [_p, _p, _p, _p, _p, _p, _p, _i, _p, _p, _p, _f, _i, _i, _i, _i,
                                  _p, _p, _i, _p, _p, _p, _sz, _p],
    "cvqpg_render_backward_workspace_size": [_i, _psz],
    "cvqpg_render_backward": [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _f, _i, _i, _i, _i,
                              _p, _p, _p, _p, _p, _p, _p, _p, _sz, _p],
    "cvqpg_render_backward_cull": [_p, _p, _p, _p, _p, _p, _p, _p, _p, _i, _p, _p, _f, _i, _i, _i, _i,
                                   _p, _p, _p, _p, _p, _p, _p, _p, _sz, _p],
    "cvqpg_blasm_tables_size": [_p, _psz],
    "cvqpg_blasm_setup": [_p, _p, _sz],
    "cvqpg_blasm_workspace_size": [_p, _psz],
    "cvqpg_blasm_forward": [_p, _p, _sz, _p, _p, _p, _sz, _p],
    "cvqpg_blasm_backward": [_p, _p, _sz, _p, _p, _p, _p, _sz, _p],
    "cvqpg_loss_workspace_size": [_p, _psz],
    "cvqpg_loss_target_range": [_p, _i, _i, _i, _i, _p, _p, _sz, _p],
    "cvqpg_loss_target_moments_size": [_p, _psz],
    "cvqpg_loss_target_moments": [_p, _p, _p, _sz, _p],
    "cvqpg_loss_forward_backward": [_p, _p, _p, _p, _p, _p, _p, _p, _p, _sz, _p],
    "cvqpg_targets_workspace_size": [_i, _i, _i, _i, _psz],
    "cvqpg_targets_synthesize": [_p, _p, _i, _i, _i, _i, _i, _f, _f, _p, _p, _p, _sz, _p],
    "cvqpg_poh_encode": [_p, _p, _sz, _p, _p, _p, _p],
    "cvqpg_gemm_bf16_tn": [_p, _i, _p, _i, _i, _i, _i, _p, _i, _p, _p],
    "cvqpg_mlp_weights_size": [_p, _psz],
    "cvqpg_mlp_workspace_size": [_p, _psz],
    "cvqpg_mlp_sync_weights": [_p, _p, _p, _sz, _p],
    "cvqpg_mlp_forward": [_p, _p, _p, _p, _p, _sz, _p, _p],
    "cvqpg_mlp_gradients": [_p, _p, _p, _p, _p, _p, _p, _p, _sz, _p, _p],
    "cvqpg_mlp_adam_step": [_p, _p, _p, _p, _p, _p, _sz, _p],
    "cvqpg_mlp_train_step": [_p, _p, _p, _p, _p, _p, _p, _p, _p, _sz, _p, _p],
    "cvqpg_fit_workspace_size": [_p, _psz],
    "cvqpg_fit_setup": [_p, _p, _p, _sz],
    "cvqpg_fit_step": [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _sz, _p],
    "cvqpg_fit_step_timed": [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _sz, _p, _p, _i],
    "cvqpg_fit_evaluate": [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _sz, _p],
    "cvqpg_fit_pair_count": [_p, _p, _sz, _p, _p],
    "cvqpg_preprocess_forward": [_p, _p, _p, _p, _p, _p, _p],
    "cvqpg_preprocess_partials": [_i],
    "cvqpg_preprocess_backward": [_p, _p, _p, _p, _p, _p, _p],
    "cvqpg_wait_probe": [_i, ctypes.c_uint, _p, _p],
}
_RESTYPES = {"cvqpg_status_string": ctypes.c_char_p}

_lib = None


def declared_symbols():
    """Every C-ABI symbol this binding knows (must match include/cvqpg.h)."""
    return sorted(_SIGNATURES)


def lib():
    """Load libcvqpg.so once; raise if it has not been built."""
    global _lib
    if _lib is None:
        # CVQPG_LIBRARY names another build of the same library (side-by-side timing of two builds)
        path = os.environ.get("CVQPG_LIBRARY", LIB_PATH)
        if not os.path.exists(path):
            raise RuntimeError(
                f"{path} is missing: build it with "
                "`python -m complex_valued_quadratic_phase_gaussian_b200.build` (needs nvcc)")
        handle = ctypes.CDLL(path)
        for name, argtypes in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.argtypes = argtypes
            fn.restype = _RESTYPES.get(name, ctypes.c_int)
        _lib = handle
    return _lib


def check(status, what):
    """Raise RuntimeError (the TORCH_CHECK surface of the reference) on a bad status."""
    if status != 0:
        msg = lib().cvqpg_status_string(status).decode()
        raise RuntimeError(f"{what}: {msg} (status {status})")


def ptr(t):
    """Device (or host) address of a tensor, or NULL for None."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_of(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def size_query(fn, *args):
    out = ctypes.c_size_t(0)
    check(fn(*args, ctypes.byref(out)), fn.__name__)
    return int(out.value)


def workspace(nbytes, device):
    """Caller-side workspace from the torch caching allocator."""
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)
