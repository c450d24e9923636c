"""Oracle: the per-tile MLP of the learned initialiser (numpy, float64).

Test infrastructure only (see oracle/__init__.py). The reference has no
learned part, so this restates the network of
complex_valued_quadratic_phase_gaussian_b200/csrc/mlp.cu in float64 with the
BF16 roundings applied at the same points as the kernels (inputs, weights,
hidden activations, back-propagated gradients), plus a rounding-free mode whose
gradients are checked against central finite differences.
"""
import numpy as np
from scipy.special import erf


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    x = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def layout(D, H, O):
    """Offsets of W1, b1, W2, b2, W3, b3 in the flat weight vector (W3/b3 padded to 128 rows)."""
    Op = (O + 127) // 128 * 128
    sizes = [("W1", (H, D)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (Op, H)), ("b3", (Op,))]
    out, o = {}, 0
    for name, shp in sizes:
        n = int(np.prod(shp))
        out[name] = (o, shp)
        o += n
    return out, o


def unpack(w, D, H, O):
    lay, _ = layout(D, H, O)
    return {k: np.asarray(w[o:o + int(np.prod(s))], dtype=np.float64).reshape(s) for k, (o, s) in lay.items()}


def pack(parts, D, H, O):
    lay, total = layout(D, H, O)
    w = np.zeros(total, dtype=np.float64)
    for k, (o, s) in lay.items():
        w[o:o + int(np.prod(s))] = np.asarray(parts[k], dtype=np.float64).ravel()
    return w


def init_weights(D, H, O, seed=0):
    """He-style init used by the learned initialiser (float32)."""
    rng = np.random.default_rng(seed)
    Op = (O + 127) // 128 * 128
    W3 = np.zeros((Op, H))
    W3[:O] = rng.normal(0, 1.0 / np.sqrt(H), (O, H)) * 0.1
    parts = dict(W1=rng.normal(0, np.sqrt(2.0 / D), (H, D)), b1=np.zeros(H), W2=rng.normal(0, np.sqrt(2.0 / H), (H, H)),
                 b2=np.zeros(H), W3=W3, b3=np.zeros(Op))
    return pack(parts, D, H, O).astype(np.float32)


def forward_backward(w, X, T, wout, D, H, O, rounding=True):
    """Loss, output Y [M,O] and flat gradient of the weighted MSE (same layout as w)."""
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    p = unpack(w, D, H, O)
    M = X.shape[0]
    X0 = r(X).astype(np.float64)
    W1, W2, W3 = (r(p[k].astype(np.float32) if rounding else p[k]).astype(np.float64) for k in ("W1", "W2", "W3"))
    W3 = W3[:O]
    Z1 = X0 @ W1.T + p["b1"]
    H1 = r(gelu(Z1).astype(np.float32) if rounding else gelu(Z1)).astype(np.float64)
    Z2 = H1 @ W2.T + p["b2"]
    H2 = r(gelu(Z2).astype(np.float32) if rounding else gelu(Z2)).astype(np.float64)
    Y = H2 @ W3.T + p["b3"][:O]
    res = Y - T
    loss = float((wout[None, :] * res * res).sum() / M)
    dY = 2.0 * wout[None, :] * res / M
    dZ3 = r(dY.astype(np.float32) if rounding else dY).astype(np.float64)
    dH2 = dZ3 @ W3
    dZ2 = dH2 * gelu_grad(Z2)
    dZ2 = r(dZ2.astype(np.float32) if rounding else dZ2).astype(np.float64)
    dH1 = dZ2 @ W2
    dZ1 = dH1 * gelu_grad(Z1)
    dZ1 = r(dZ1.astype(np.float32) if rounding else dZ1).astype(np.float64)
    Op = (O + 127) // 128 * 128
    gW3 = np.zeros((Op, H))
    gW3[:O] = dZ3.T @ H2
    gb3 = np.zeros(Op)
    gb3[:O] = dZ3.sum(0)
    grads = dict(W1=dZ1.T @ X0, b1=dZ1.sum(0), W2=dZ2.T @ H1, b2=dZ2.sum(0), W3=gW3, b3=gb3)
    return loss, Y, pack(grads, D, H, O)


def adam_step(w, m1, m2, g, t, lr, b1=0.9, b2=0.999, eps=1e-8, valid_mask=None):
    """One bias-corrected Adam step (t counts from 1); returns new (w, m1, m2)."""
    m1 = b1 * m1 + (1 - b1) * g
    m2 = b2 * m2 + (1 - b2) * g * g
    w = w - lr * (m1 / (1 - b1 ** t)) / (np.sqrt(m2 / (1 - b2 ** t)) + eps)
    if valid_mask is not None:
        w = np.where(valid_mask, w, 0.0)
    return w, m1, m2


def valid_mask(D, H, O):
    """True for weights that train (the padding rows of W3/b3 stay zero)."""
    lay, total = layout(D, H, O)
    mask = np.ones(total, dtype=bool)
    o, (rows, cols) = lay["W3"][0], lay["W3"][1]
    mask[o + O * cols:o + rows * cols] = False
    o, (rows,) = lay["b3"][0], lay["b3"][1]
    mask[o + O:o + rows] = False
    return mask
