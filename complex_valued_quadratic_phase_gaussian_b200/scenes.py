"""Seeded synthetic scenes and multi-plane targets for the fit.

The reference fits photographs from its data/ folder; the workloads here are
seeded synthetic scenes of the same shapes:

* ``grayscale_blobs``: target = sum of isotropic Gaussian blobs normalised to
  [0, 1]; depth = smooth ramp plus blobs.
* ``rgb_blobs``: target = coloured anisotropic Gaussian blobs plus 1/f noise;
  depth = a smooth 1/f field.

``multiplane_targets`` turns (image, depth) into the per-plane defocus targets
and the per-pixel plane index exactly as the reference loss does
(utils/propagator.py:361-415 with the factory settings of
utils/data_utils.py:66-82: 21-tap kernels, sigma = int(|i-j| * 8), the
in-focus kernel an impulse). It is one-off data preparation, not part of the
iteration.
"""
import math

import numpy as np
import torch
import torch.nn.functional as F

from . import _lib


def _fbm(rng, H, W, beta=1.0):
    """1/f^beta noise field in [0, 1] (spectral synthesis, seeded)."""
    fy = np.fft.fftfreq(H)[:, None]
    fx = np.fft.rfftfreq(W)[None, :]
    f = np.sqrt(fx * fx + fy * fy)
    f[0, 0] = 1.0
    amp = 1.0 / f ** beta
    amp[0, 0] = 0.0
    spec = amp * (rng.normal(size=amp.shape) + 1j * rng.normal(size=amp.shape))
    field = np.fft.irfft2(spec, s=(H, W))
    field -= field.min()
    return field / max(field.max(), 1e-12)


def grayscale_blobs(H, W, seed=0, num_blobs=64):
    """256x256-style grayscale target (64 isotropic blobs) and depth (ramp + blobs)."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float64)
    img = np.zeros((H, W))
    for _ in range(num_blobs):
        cx, cy = rng.uniform(0, W), rng.uniform(0, H)
        s = rng.uniform(0.02, 0.08) * min(H, W)
        img += rng.uniform(0.3, 1.0) * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * s * s))
    img = (img - img.min()) / max(img.max() - img.min(), 1e-12)
    depth = 0.6 * (xx / max(W - 1, 1)) + 0.2 * (yy / max(H - 1, 1))
    for _ in range(6):
        cx, cy = rng.uniform(0, W), rng.uniform(0, H)
        s = rng.uniform(0.05, 0.15) * min(H, W)
        depth += 0.25 * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * s * s))
    depth = (depth - depth.min()) / max(depth.max() - depth.min(), 1e-12)
    return img[None].astype(np.float32), depth.astype(np.float32)


def rgb_blobs(H, W, seed=0, num_blobs=2000, scale=None):
    """1080p-style RGB target (coloured anisotropic blobs + 1/f noise) and a smooth 1/f depth.

    ``scale`` sets the blob size unit in pixels (default min(H, W)); a crop with
    the statistics of a 1080p scene uses scale=1080 and num_blobs scaled by area.
    """
    rng = np.random.default_rng(seed)
    img = np.zeros((3, H, W))
    scale = min(H, W) if scale is None else scale
    for _ in range(num_blobs):
        cx, cy = rng.uniform(0, W), rng.uniform(0, H)
        sx, sy = rng.uniform(0.004, 0.03, 2) * scale
        th = rng.uniform(0, math.pi)
        col = rng.uniform(0, 1, 3)
        r = int(4 * max(sx, sy)) + 1
        x0, x1 = max(0, int(cx) - r), min(W, int(cx) + r + 1)
        y0, y1 = max(0, int(cy) - r), min(H, int(cy) + r + 1)
        if x0 >= x1 or y0 >= y1:
            continue
        yy, xx = np.mgrid[y0:y1, x0:x1].astype(np.float64)
        dx, dy = xx - cx, yy - cy
        u = dx * math.cos(th) + dy * math.sin(th)
        v = -dx * math.sin(th) + dy * math.cos(th)
        g = np.exp(-0.5 * (u * u / (sx * sx) + v * v / (sy * sy)))
        img[:, y0:y1, x0:x1] += col[:, None, None] * g[None]
    for c in range(3):
        img[c] += 0.35 * _fbm(rng, H, W, 1.0)
    img -= img.min()
    img /= max(img.max(), 1e-12)
    depth = _fbm(rng, H, W, 2.0)
    return img.astype(np.float32), depth.astype(np.float32)


def rgb_crop_like_1080p(H, W, seed=0):
    """An H x W scene with the per-pixel statistics of ``rgb_blobs(1080, 1920)`` (blob sizes and density)."""
    n = max(1, int(round(2000 * H * W / (1080.0 * 1920.0))))
    return rgb_blobs(H, W, seed=seed, num_blobs=n, scale=1080)


def _gaussian_kernel_2d(length, sigma):
    x = torch.linspace(-length / 2.0, length / 2.0, length, dtype=torch.float64)
    s = float(sigma) if sigma != 0 else 1e-5
    X, Y = torch.meshgrid(x, x, indexing="ij")
    k = 1.0 / (2.0 * math.pi * s * s) * torch.exp(-(X ** 2 / (2.0 * s ** 2) + Y ** 2 / (2.0 * s ** 2)))
    return k / k.sum()


def multiplane_targets(image, depth, num_planes, blur_size=20, blur_ratio=8, split_ratio=1.0, device="cpu"):
    """Per-plane defocus targets [P,C,H,W] (float32) and plane index [H,W] (uint8)."""
    img = torch.as_tensor(image, dtype=torch.float32, device=device)
    C, H, W = img.shape
    d = torch.as_tensor(depth, dtype=torch.float32, device=device).reshape(H, W)
    ratio = split_ratio if num_planes == 2 else 1.0
    q = torch.round(torch.pow(d, ratio) * (num_planes - 1))
    L = blur_size + 1 if blur_size % 2 == 0 else blur_size
    targets = torch.zeros(num_planes, C, H, W, dtype=torch.float32, device=device)
    masks = [(q == j).float() for j in range(num_planes)]
    blurred = {}
    for ch in range(C):
        full = img[ch]
        for i in range(num_planes):
            acc = torch.zeros(H, W, dtype=torch.float32, device=device)
            for j in range(num_planes):
                if float((full * masks[j]).sum()) > 0:
                    sig = 0 if i == j else int(abs(i - j) * blur_ratio)
                    key = (ch, sig)
                    if key not in blurred:
                        k = _gaussian_kernel_2d(L, sig).float().to(device)[None, None]
                        blurred[key] = F.conv2d(full[None, None], k, padding="same")[0, 0]
                    acc = acc + blurred[key] * masks[j]
            targets[i, ch] = acc
    return targets.contiguous(), q.to(torch.uint8).contiguous()


def multiplane_targets_device(image, depth, num_planes, blur_size=20, blur_ratio=8, split_ratio=1.0, device="cuda"):
    """Per-plane defocus targets [P,C,H,W] and plane index [H,W] with the library's kernels
    (cvqpg_targets_synthesize): the same arithmetic as ``multiplane_targets``, on the GPU."""
    dev = torch.device(device)
    img = torch.as_tensor(image, dtype=torch.float32).to(dev).contiguous()
    C, H, W = img.shape
    d = torch.as_tensor(depth, dtype=torch.float32).to(dev).reshape(H, W).contiguous()
    targets = torch.empty((num_planes, C, H, W), dtype=torch.float32, device=dev)
    q = torch.empty((H, W), dtype=torch.uint8, device=dev)
    lib = _lib.lib()
    ws = _lib.workspace(_lib.size_query(lib.cvqpg_targets_workspace_size, C, H, W, int(num_planes)), dev)
    _lib.check(lib.cvqpg_targets_synthesize(_lib.ptr(img), _lib.ptr(d), C, H, W, int(num_planes), int(blur_size),
                                            float(blur_ratio), float(split_ratio), _lib.ptr(targets), _lib.ptr(q),
                                            _lib.ptr(ws), ws.numel(), _lib.stream_of(dev)), "cvqpg_targets_synthesize")
    return targets, q
