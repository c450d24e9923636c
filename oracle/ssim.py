"""SSIM restatement -- TEST INFRASTRUCTURE ONLY.

The reference computes its SSIM loss with the third-party package
pytorch_msssim 1.0.0 (utils/data_utils.py:7, 39, 61), which is not installed
here; this module restates SSIM from Z. Wang, A. C. Bovik, H. R. Sheikh and
E. P. Simoncelli, "Image quality assessment: from error visibility to
structural similarity", IEEE TIP 13(4), 2004, with that package's documented
defaults: 11-tap Gaussian window, sigma 1.5, K = (0.01, 0.03), data_range 1,
separable filtering without padding ("valid"), mean over the map, then over
channels and batch. Parity for SSIM is therefore UNPINNED.

``SSIMModule`` is a torch module (installed as ``pytorch_msssim.SSIM`` when the
golden fixtures are generated); ``ssim_value_and_grad`` is the float64 numpy
oracle with the analytic gradient with respect to the first image.
"""
import numpy as np
import torch
import torch.nn.functional as F

WIN = 11
SIGMA = 1.5
K1, K2 = 0.01, 0.03


def gauss_window_1d(size=WIN, sigma=SIGMA):
    coords = np.arange(size, dtype=np.float64) - size // 2
    g = np.exp(-(coords ** 2) / (2.0 * sigma ** 2))
    return g / g.sum()


def _filter_valid_torch(x, w1):
    C = x.shape[1]
    wx = w1.view(1, 1, 1, -1).repeat(C, 1, 1, 1)
    wy = w1.view(1, 1, -1, 1).repeat(C, 1, 1, 1)
    out = x
    if out.shape[-1] >= w1.numel():
        out = F.conv2d(out, wx, groups=C)
    if out.shape[-2] >= w1.numel():
        out = F.conv2d(out, wy, groups=C)
    return out


def ssim_torch(X, Y, data_range=1.0, win_size=WIN, win_sigma=SIGMA, K=(K1, K2)):
    w1 = torch.tensor(gauss_window_1d(win_size, win_sigma), dtype=X.dtype, device=X.device)
    C1 = (K[0] * data_range) ** 2
    C2 = (K[1] * data_range) ** 2
    mu1 = _filter_valid_torch(X, w1)
    mu2 = _filter_valid_torch(Y, w1)
    s11 = _filter_valid_torch(X * X, w1) - mu1 * mu1
    s22 = _filter_valid_torch(Y * Y, w1) - mu2 * mu2
    s12 = _filter_valid_torch(X * Y, w1) - mu1 * mu2
    cs_map = (2 * s12 + C2) / (s11 + s22 + C2)
    ssim_map = ((2 * mu1 * mu2 + C1) / (mu1 * mu1 + mu2 * mu2 + C1)) * cs_map
    return torch.flatten(ssim_map, 2).mean(-1)  # [B, C]


class SSIMModule(torch.nn.Module):
    def __init__(self, data_range=255, size_average=True, win_size=WIN, win_sigma=SIGMA, channel=3,
                 spatial_dims=2, K=(K1, K2), nonnegative_ssim=False):
        super().__init__()
        self.data_range, self.size_average = data_range, size_average
        self.win_size, self.win_sigma, self.K = win_size, win_sigma, K
        self.nonnegative_ssim = nonnegative_ssim

    def forward(self, X, Y):
        s = ssim_torch(X, Y, self.data_range, self.win_size, self.win_sigma, self.K)
        if self.nonnegative_ssim:
            s = torch.relu(s)
        return s.mean() if self.size_average else s.mean(1)


def _filt_valid_np(x, w):
    """x [..., H, W] -> [..., H-10, W-10] separable valid correlation (float64)."""
    L = w.size
    H, W = x.shape[-2], x.shape[-1]
    t = np.zeros(x.shape[:-1] + (W - L + 1,))
    for i in range(L):
        t += w[i] * x[..., i:i + W - L + 1]
    o = np.zeros(x.shape[:-2] + (H - L + 1, W - L + 1))
    for i in range(L):
        o += w[i] * t[..., i:i + H - L + 1, :]
    return o


def _filt_full_np(m, w, H, W):
    """Adjoint of _filt_valid_np: map [.., H-10, W-10] back to [.., H, W]."""
    L = w.size
    t = np.zeros(m.shape[:-2] + (H, m.shape[-1]))
    for i in range(L):
        t[..., i:i + m.shape[-2], :] += w[i] * m
    o = np.zeros(m.shape[:-2] + (H, W))
    for i in range(L):
        o[..., :, i:i + m.shape[-1]] += w[i] * t
    return o


def ssim_value_and_grad(X, Y, data_range=1.0):
    """Mean SSIM over [C,H,W] images (float64) and dSSIM/dX."""
    X = np.asarray(X, dtype=np.float64)
    Y = np.asarray(Y, dtype=np.float64)
    w = gauss_window_1d()
    C1 = (K1 * data_range) ** 2
    C2 = (K2 * data_range) ** 2
    H, W = X.shape[-2], X.shape[-1]
    mu1, mu2 = _filt_valid_np(X, w), _filt_valid_np(Y, w)
    exx, eyy, exy = _filt_valid_np(X * X, w), _filt_valid_np(Y * Y, w), _filt_valid_np(X * Y, w)
    s11, s22, s12 = exx - mu1 ** 2, eyy - mu2 ** 2, exy - mu1 * mu2
    A1, A2 = 2 * mu1 * mu2 + C1, 2 * s12 + C2
    B1, B2 = mu1 ** 2 + mu2 ** 2 + C1, s11 + s22 + C2
    ssim_map = (A1 * A2) / (B1 * B2)
    n = ssim_map[0].size * X.shape[0]
    val = ssim_map.mean()
    # d ssim_map / d(mu1, exx, exy)
    d_mu1 = (2 * mu2 * A2 / (B1 * B2) - 2 * mu1 * A1 * A2 / (B1 ** 2 * B2)
             + A1 / B1 * (-2 * mu2 / B2 + 2 * mu1 * A2 / B2 ** 2))
    d_exx = -A1 * A2 / (B1 * B2 ** 2)
    d_exy = 2 * A1 / (B1 * B2)
    g = (_filt_full_np(d_mu1, w, H, W) + 2 * X * _filt_full_np(d_exx, w, H, W)
         + Y * _filt_full_np(d_exy, w, H, W)) / n
    return val, g
