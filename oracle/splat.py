"""Oracle: tile binning and the complex quadratic-phase splat (numpy, float64).

Test infrastructure only (see oracle/__init__.py).

* ``bin_lists`` restates the reference binning: getRect + preprocess +
  duplicateWithKeys + 64-bit CUB sort + identifyTileRanges
  (cuda/forward.cu:8-60, cuda/raster.cu:60-95) for the CUDA rule, and the torch
  renderer's per-64-px-tile 3-sigma circle test (model_2d_gaussian_rgb.py:311-314,
  400-406). Rectangle/threshold arithmetic is emulated in float32 with the
  reference operation order, so the lists are exact.
* ``splat_forward`` restates renderTileKernel (cuda/forward.cu:63-162) /
  qpf_render_reference (cuda/rasterizer.py:74-91) in float64.
* ``splat_backward`` restates renderBackwardKernel (cuda/backward.cu:22-168),
  including both paths of dL/dmahal (cuda/backward.cu:131-138), in float64.
"""
import numpy as np

CULL_CUDA16_5SIGMA = 0
CULL_TORCH64_3SIGMA = 1
CULL_NONE = 2

F32 = np.float32


def list_grid(cull, W, H):
    if cull == CULL_CUDA16_5SIGMA:
        return 16, (W + 15) // 16, (H + 15) // 16
    if cull == CULL_TORCH64_3SIGMA:
        return 64, (W + 63) // 64, (H + 63) // 64
    return 0, 1, 1


def tile_rect_f32(mx, my, r, gx, gy):
    """Reference getRect (cuda/forward.cu:8-13), float32 op order."""
    mx = F32(mx)
    my = F32(my)
    fr = F32(r)
    sixteen = F32(16.0)

    def clampi(v, hi):
        return int(min(hi, max(0, int(np.trunc(v)))))

    x0 = clampi(F32(mx - fr) / sixteen, gx)
    y0 = clampi(F32(my - fr) / sixteen, gy)
    x1 = clampi(F32(F32(F32(mx + fr) + sixteen) - F32(1.0)) / sixteen, gx)
    y1 = clampi(F32(F32(F32(my + fr) + sixteen) - F32(1.0)) / sixteen, gy)
    return x0, y0, x1, y1


def _tiles_of(g, cull, means, W, H, radii, radius3, lgx, lgy):
    mx, my = F32(means[g, 0]), F32(means[g, 1])
    if cull == CULL_CUDA16_5SIGMA:
        r = int(radii[g])
        if r <= 0:
            return []
        x0, y0, x1, y1 = tile_rect_f32(mx, my, r, lgx, lgy)
        return [y * lgx + x for y in range(y0, y1) for x in range(x0, x1)]
    if cull == CULL_TORCH64_3SIGMA:
        thr = F32(F32(radius3[g]) + F32(45.254833995939045))
        thr2 = F32(thr * thr)
        out = []
        for ty in range(lgy):
            y0 = ty * 64
            y1 = min(y0 + 64, H)
            cy = F32((y0 + y1) / 2.0)
            dy = F32(my - cy)
            dy2 = F32(dy * dy)
            for tx in range(lgx):
                x0 = tx * 64
                x1 = min(x0 + 64, W)
                cx = F32((x0 + x1) / 2.0)
                dx = F32(mx - cx)
                d2 = F32(F32(dx * dx) + dy2)
                if d2 < thr2:
                    out.append(ty * lgx + tx)
        return out
    return [0]


def bin_lists(means, W, H, cull=CULL_CUDA16_5SIGMA, radii=None, radius3=None):
    """Exact per-tile Gaussian lists. Returns (point_list int32, ranges int32 [L,2])."""
    means = np.asarray(means, dtype=np.float32)
    n = means.shape[0]
    _, lgx, lgy = list_grid(cull, W, H)
    keys, vals = [], []
    for g in range(n):
        for t in _tiles_of(g, cull, means, W, H, radii, radius3, lgx, lgy):
            keys.append(t)
            vals.append(g)
    keys = np.asarray(keys, dtype=np.int64)
    vals = np.asarray(vals, dtype=np.int64)
    ranges = np.zeros((lgx * lgy, 2), dtype=np.int32)
    if keys.size == 0:
        return np.zeros(1, dtype=np.int32), ranges
    # 64-bit key (tile << 32 | id) sort == stable sort on tile of id-ordered pairs
    order = np.argsort((keys << 32) | vals, kind="stable")
    ks = keys[order]
    point_list = vals[order].astype(np.int32)
    # identifyTileRangesKernel (cuda/forward.cu:49-60)
    starts = np.flatnonzero(np.r_[True, ks[1:] != ks[:-1]])
    ends = np.r_[starts[1:], ks.size]
    for s, e in zip(starts, ends):
        ranges[ks[s]] = (s, e)
    return point_list, ranges


def _list_index(cull, tx, ty, lgx):
    if cull == CULL_CUDA16_5SIGMA:
        return ty * lgx + tx
    if cull == CULL_TORCH64_3SIGMA:
        return (ty // 4) * lgx + (tx // 4)
    return 0


def _tile_pixels(tx, ty, W, H):
    xs = np.arange(tx * 16, min(tx * 16 + 16, W), dtype=np.float64)
    ys = np.arange(ty * 16, min(ty * 16 + 16, H), dtype=np.float64)
    yy, xx = np.meshgrid(ys, xs, indexing="ij")
    return xx.ravel(), yy.ravel()


def _as64(*arrs):
    return [np.asarray(a, dtype=np.float64) for a in arrs]


def splat_forward(means, inv_cov, colours, phase, opac, curv, area, k, dxy2, W, H, cull=CULL_NONE,
                  point_list=None, ranges=None, chunk=512, phase_iso=False):
    """Complex field [C,H,W] (complex128). With cull=CULL_NONE every Gaussian hits every pixel.

    phase_iso: the isotropic quadratic phase 0.5 c |r - mu|^2 dxy2 of the torch
    renderer's --phase_iso (model_2d_gaussian_rgb.py:356-359) instead of the
    Mahalanobis form 0.5 c m area dxy2 (model_2d_gaussian_rgb.py:360-363)."""
    means, inv_cov, colours, phase, opac, curv, area, k = _as64(means, inv_cov, colours, phase, opac, curv, area, k)
    C = colours.shape[1]
    n = means.shape[0]
    out = np.zeros((C, H, W), dtype=np.complex128)
    _, lgx, _ = list_grid(cull, W, H)
    for ty in range((H + 15) // 16):
        for tx in range((W + 15) // 16):
            if cull == CULL_NONE:
                ids = np.arange(n)
            else:
                s, e = ranges[_list_index(cull, tx, ty, lgx)]
                ids = np.asarray(point_list[s:e], dtype=np.int64)
            if ids.size == 0:
                continue
            px, py = _tile_pixels(tx, ty, W, H)
            acc = np.zeros((C, px.size), dtype=np.complex128)
            for c0 in range(0, ids.size, chunk):
                g = ids[c0:c0 + chunk]
                dx = means[g, 0:1] - px[None, :]
                dy = means[g, 1:2] - py[None, :]
                i00, i01, i11 = inv_cov[g, 0:1], inv_cov[g, 1:2], inv_cov[g, 2:3]
                mahal = dx * (i00 * dx + i01 * dy) + dy * (i01 * dx + i11 * dy)
                G = np.exp(np.maximum(-0.5 * mahal, -50.0))
                alpha = opac[g, None] * G
                if phase_iso:
                    base = 0.5 * curv[g, None] * (dx * dx + dy * dy) * dxy2
                else:
                    base = 0.5 * curv[g, None] * mahal * area[g, None] * dxy2
                for c in range(C):
                    ph = phase[g, c:c + 1] + k[c] * base
                    acc[c] += np.sum(colours[g, c:c + 1] * alpha * np.exp(1j * ph), axis=0)
            y0, x0 = ty * 16, tx * 16
            hh, ww = min(16, H - y0), min(16, W - x0)
            out[:, y0:y0 + hh, x0:x0 + ww] = acc.reshape(C, hh, ww)
    return out


def splat_backward(grad, means, inv_cov, colours, phase, opac, curv, area, k, dxy2, W, H, cull=CULL_NONE,
                   point_list=None, ranges=None, chunk=512, phase_iso=False):
    """Gradients (d_means, d_inv, d_col, d_ph, d_op, d_cv, d_ar) in float64.

    grad is dL/dU as complex (real part dL/dRe, imaginary part dL/dIm).
    """
    means, inv_cov, colours, phase, opac, curv, area, k = _as64(means, inv_cov, colours, phase, opac, curv, area, k)
    grad = np.asarray(grad, dtype=np.complex128)
    C = colours.shape[1]
    n = means.shape[0]
    d_means = np.zeros((n, 2))
    d_inv = np.zeros((n, 3))
    d_col = np.zeros((n, C))
    d_ph = np.zeros((n, C))
    d_op = np.zeros(n)
    d_cv = np.zeros(n)
    d_ar = np.zeros(n)
    _, lgx, _ = list_grid(cull, W, H)
    for ty in range((H + 15) // 16):
        for tx in range((W + 15) // 16):
            if cull == CULL_NONE:
                ids = np.arange(n)
            else:
                s, e = ranges[_list_index(cull, tx, ty, lgx)]
                ids = np.asarray(point_list[s:e], dtype=np.int64)
            if ids.size == 0:
                continue
            px, py = _tile_pixels(tx, ty, W, H)
            y0, x0 = ty * 16, tx * 16
            hh, ww = min(16, H - y0), min(16, W - x0)
            gp = grad[:, y0:y0 + hh, x0:x0 + ww].reshape(C, -1)
            for c0 in range(0, ids.size, chunk):
                g = ids[c0:c0 + chunk]
                dx = means[g, 0:1] - px[None, :]
                dy = means[g, 1:2] - py[None, :]
                i00, i01, i11 = inv_cov[g, 0:1], inv_cov[g, 1:2], inv_cov[g, 2:3]
                mahal = dx * (i00 * dx + i01 * dy) + dy * (i01 * dx + i11 * dy)
                raw_power = -0.5 * mahal
                G = np.exp(np.maximum(raw_power, -50.0))
                o = opac[g, None]
                alpha = o * G
                cv = curv[g, None]
                ar = area[g, None]
                d2 = dx * dx + dy * dy
                base = 0.5 * cv * d2 * dxy2 if phase_iso else 0.5 * cv * mahal * ar * dxy2
                S_alpha = np.zeros_like(mahal)
                S_base = np.zeros_like(mahal)
                for c in range(C):
                    ph = phase[g, c:c + 1] + k[c] * base
                    s, co = np.sin(ph), np.cos(ph)
                    gr, gi = gp[c].real[None, :], gp[c].imag[None, :]
                    proj_c = gr * co + gi * s
                    proj_s = -gr * s + gi * co
                    A = colours[g, c:c + 1]
                    d_col[g, c] += np.sum(alpha * proj_c, axis=1)
                    dph = A * alpha * proj_s
                    d_ph[g, c] += np.sum(dph, axis=1)
                    S_alpha += A * proj_c
                    S_base += k[c] * dph
                dpow = np.where(raw_power >= -50.0, -0.5, 0.0)
                if phase_iso:
                    dmahal = S_alpha * o * G * dpow
                    d_cv[g] += np.sum(S_base * 0.5 * d2 * dxy2, axis=1)
                    # the phase depends on the means directly: dbase/dmu = c dxy2 (mu - r)
                    d_means[g, 0] += np.sum(S_base * cv * dxy2 * dx, axis=1)
                    d_means[g, 1] += np.sum(S_base * cv * dxy2 * dy, axis=1)
                else:
                    dmahal = S_alpha * o * G * dpow + S_base * 0.5 * cv * ar * dxy2
                    d_cv[g] += np.sum(S_base * 0.5 * mahal * ar * dxy2, axis=1)
                    d_ar[g] += np.sum(S_base * 0.5 * cv * mahal * dxy2, axis=1)
                d_inv[g, 0] += np.sum(dmahal * dx * dx, axis=1)
                d_inv[g, 1] += np.sum(dmahal * 2.0 * dx * dy, axis=1)
                d_inv[g, 2] += np.sum(dmahal * dy * dy, axis=1)
                d_means[g, 0] += np.sum(dmahal * 2.0 * (i00 * dx + i01 * dy), axis=1)
                d_means[g, 1] += np.sum(dmahal * 2.0 * (i11 * dy + i01 * dx), axis=1)
                d_op[g] += np.sum(S_alpha * G, axis=1)
    return d_means, d_inv, d_col, d_ph, d_op, d_cv, d_ar


def radius5_int(cov00, cov01, cov11):
    """Reference CUDA culling radius (model_2d_gaussian_rgb.py:433-436), float32 torch ops."""
    cov00, cov01, cov11 = (np.asarray(a, dtype=np.float32) for a in (cov00, cov01, cov11))
    mid = F32(0.5) * (cov00 + cov11)
    disc = np.sqrt(((cov00 - cov11) * F32(0.5)) ** 2 + cov01 ** 2)
    return np.ceil(F32(5.0) * np.sqrt(mid + disc)).astype(np.int32)


def radius3_float(cov00, cov01, cov11):
    """Reference torch-renderer culling radius (model_2d_gaussian_rgb.py:401-403), float32."""
    cov00, cov01, cov11 = (np.asarray(a, dtype=np.float32) for a in (cov00, cov01, cov11))
    mid = F32(0.5) * (cov00 + cov11)
    disc = np.sqrt(((cov00 - cov11) * F32(0.5)) ** 2 + cov01 ** 2)
    return (F32(3.0) * np.sqrt(mid + disc)).astype(np.float32)
