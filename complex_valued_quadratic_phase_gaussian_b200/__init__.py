"""B200-native (sm_100a) CVQPG hologram-fitting kernels behind the reference API.

Drop-in names (reference ``cuda/__init__.py``): ``qpf_render``. The kernels live
in ``libcvqpg.so`` (C ABI, include/cvqpg.h), loaded through ctypes.
"""
from .rasterizer import QPFRender, qpf_render, qpf_render_cull, ext  # noqa: F401
from .build import build  # noqa: F401

__all__ = ["QPFRender", "qpf_render", "qpf_render_cull", "ext", "build"]
