"""Oracle: multi-plane loss with SSIM, its gradient, and the target noise (numpy).

Test infrastructure only (see oracle/__init__.py). Restates

* multiplane_loss_odak.__call__      utils/propagator.py:417-449
* GaussianLoss (0.025 * 0.2 * (1 - SSIM))  utils/data_utils.py:22-41
* the per-plane loop of the fit      train_2d_gaussian_rgb.py:192-199
* set_targets / add_defocus_blur     utils/propagator.py:361-415 (target synthesis)

The noise generator restates the kernels' Philox4x32-10 + Box-Muller
(J. K. Salmon et al., SC 2011) so the noisy loss can be compared exactly.
"""
import numpy as np

from . import ssim as ossim

M32 = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised Philox4x32-10 on uint64 arrays holding 32-bit values."""
    c = [np.asarray(x, dtype=np.uint64) & M32 for x in (c0, c1, c2, c3)]
    k0 = np.uint64(k0) & M32
    k1 = np.uint64(k1) & M32
    M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
    W0, W1 = np.uint64(0x9E3779B9), np.uint64(0xBB67AE85)
    for _ in range(10):
        p0 = M0 * c[0]
        p1 = M1 * c[2]
        hi0, lo0 = (p0 >> np.uint64(32)) & M32, p0 & M32
        hi1, lo1 = (p1 >> np.uint64(32)) & M32, p1 & M32
        c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
        k0 = (k0 + W0) & M32
        k1 = (k1 + W1) & M32
    return c


def normals4_at(seed, offset, q):
    """Four standard normals per counter q of stream (seed, offset): float32 Box-Muller on the
    Philox word pairs (w0, w1) and (w2, w3). Returns float32 [..., 4]."""
    q = np.asarray(q, dtype=np.uint64)
    seed, offset = int(seed), int(offset)
    r = philox4x32_10(q & M32, q >> np.uint64(32), offset & 0xFFFFFFFF, (offset >> 32) & 0xFFFFFFFF,
                      seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    u = [((w.astype(np.float64) + 1.0) * 2.3283064365386963e-10).astype(np.float32) for w in r]
    two_pi = np.float32(2.0 * np.pi)
    r01 = np.sqrt(np.float32(-2.0) * np.log(u[0]))
    r23 = np.sqrt(np.float32(-2.0) * np.log(u[2]))
    a1, a3 = two_pi * u[1], two_pi * u[3]
    return np.stack([r01 * np.cos(a1), r01 * np.sin(a1), r23 * np.cos(a3), r23 * np.sin(a3)], -1).astype(np.float32)


def plane_noise(shape, seed, iteration):
    """Noise tensor [P,C,H,W] for one iteration.

    Element (image i = p*C + c, row y, column x) takes normal (y % 4) of counter
    q = (i * ceil(H/4) + y // 4) * W + x, so four vertically adjacent pixels
    share one Philox call.
    """
    P, C, H, W = shape
    Hq = (H + 3) // 4
    q = np.arange(P * C * Hq * W, dtype=np.uint64)
    n4 = normals4_at(seed, iteration, q).reshape(P * C, Hq, W, 4)
    z = n4.transpose(0, 1, 3, 2).reshape(P * C, Hq * 4, W)[:, :H, :]
    return np.ascontiguousarray(z).reshape(P, C, H, W)


def multiplane_loss_pred(pred, targets, depth_plane, weights=(1.0, 1.0, 1.0), ssim_weight=0.005, noise=None,
                         noise_ratio=1e-3):
    """Loss over all planes of the clamped intensity pred [P,C,H,W] and dL/d(pred).

    noise: None (no injection) or standard normals [P,C,H,W].
    Returns (loss, per-plane MSE, per-plane SSIM, per-plane loss, grad_pred).
    """
    pred = np.asarray(pred, dtype=np.float64)
    T = np.asarray(targets, dtype=np.float64)
    P, C, H, W = pred.shape
    n = C * H * W
    w0, w1, w2 = weights
    total = 0.0
    mses, ssims, losses = [], [], []
    gx = np.zeros_like(pred)
    for p in range(P):
        x, t = pred[p], T[p]
        m = (np.asarray(depth_plane) == p).astype(np.float64)[None].repeat(C, 0)
        if noise is None:
            nt = t
        else:
            rng_ = float(np.float32(t.max()) - np.float32(t.min()))
            nt = t + (np.asarray(noise[p], dtype=np.float64) * noise_ratio) * rng_
        d0, d1, d2 = x - t, x * m - nt * m, x * nt - nt * nt
        l2 = (w0 * (d0 ** 2).sum() + w1 * (d1 ** 2).sum() + w2 * (d2 ** 2).sum()) / n
        s, gs = ossim.ssim_value_and_grad(x, t)
        lp = l2 + ssim_weight * (1.0 - s)
        total += lp
        mses.append((d0 ** 2).mean())
        ssims.append(s)
        losses.append(lp)
        gx[p] = 2.0 / n * (w0 * d0 + w1 * d1 * m + w2 * d2 * nt) - ssim_weight * gs
    return total, np.array(mses), np.array(ssims), np.array(losses), gx


def multiplane_loss(V, targets, depth_plane, weights=(1.0, 1.0, 1.0), ssim_weight=0.005, noise=None,
                    noise_ratio=1e-3):
    """Loss over all planes and dL/dV (torch convention). V [P,C,H,W] complex.

    noise: None (no injection) or standard normals [P,C,H,W].
    Returns (loss, per-plane MSE, per-plane SSIM, grad_V).
    """
    V = np.asarray(V, dtype=np.complex128)
    I = np.abs(V) ** 2
    total, mses, ssims, _, gx = multiplane_loss_pred(np.clip(I, 0.0, 1.0), targets, depth_plane, weights,
                                                     ssim_weight, noise, noise_ratio)
    gI = np.where(I <= 1.0, gx, 0.0)
    gV = 2.0 * V * gI
    return total, mses, ssims, gV


def quantise_depth(depth, num_planes, split_ratio=1.0):
    """set_targets depth slicing (utils/propagator.py:365-372): round(depth^r * (P-1)), half to even."""
    ratio = split_ratio if num_planes == 2 else 1.0
    return np.round(np.power(np.asarray(depth, dtype=np.float32), np.float32(ratio)) * np.float32(num_planes - 1))


def gaussian_kernel_2d(length, sigma):
    x = np.linspace(-length / 2.0, length / 2.0, length)
    s = float(sigma) if sigma != 0 else 1e-5
    X, Y = np.meshgrid(x, x, indexing="ij")
    k = 1.0 / (2.0 * np.pi * s * s) * np.exp(-(X ** 2 / (2.0 * s ** 2) + Y ** 2 / (2.0 * s ** 2)))
    return k / k.sum()


def defocus_targets(image, depth, num_planes, blur_size=20, blur_ratio=8, split_ratio=1.0):
    """Multi-plane targets and plane index (utils/propagator.py:361-415, utils/data_utils.py:66-82)."""
    from scipy.signal import correlate2d
    image = np.asarray(image, dtype=np.float64)
    C, H, W = image.shape
    L = blur_size + 1 if blur_size % 2 == 0 else blur_size
    q = quantise_depth(depth, num_planes, split_ratio).reshape(H, W)
    targets = np.zeros((num_planes, C, H, W))
    for ch in range(C):
        full = image[ch]
        for i in range(num_planes):
            acc = np.zeros((H, W))
            for j in range(num_planes):
                mj = (q == j).astype(np.float64)
                if (full * mj).sum() > 0:
                    sig = 0 if i == j else int(abs(i - j) * blur_ratio)
                    k = gaussian_kernel_2d(L, sig)
                    acc += correlate2d(full, k, mode="same", boundary="fill") * mj
            targets[i, ch] = acc
    return targets, q.astype(np.uint8)
