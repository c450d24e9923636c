"""Learned initialiser: predict a fit's starting Gaussians tile by tile.

The reference starts every fit from random Gaussians
(model_2d_gaussian_rgb.py:41-77); that stays the fallback here. The learned
path cuts the image into 16x16 tiles and asks a small MLP (mlp.TileMLP, on the
tensor cores) for 12 Gaussians per tile:

* input, 1024 values per tile: the tile's RGB image (3 x 16 x 16) and its depth
  (16 x 16), zero outside the image;
* output, 156 = 12 slots x 13 raw parameters per tile, slot s being
  [u, v, scale_x, scale_y, rotation, colour RGB, phase RGB, opacity, curvature]
  with (u, v) the mean in tile units relative to the tile's corner, the others in
  the reference's raw (pre-activation) parameterisation; rotation is wrapped to
  [0, pi) and phase to [0, 2 pi) (their activations are periodic).

Training pairs come from fits that start from ``grid_init``: slot s of every
tile starts at the same place in its tile, so after the fit slot s of a tile is
still "its" Gaussian and the converged parameters are a consistent regression
target. ``make_pairs`` runs those fits with the batched fitter; ``train`` fits
the MLP with Adam on the GPU; ``learned_init`` turns a prediction into a raw
parameter set for ``Fitter``.
"""
import math
import time

import numpy as np
import torch

from .batch import BatchedFitter, FitJob
from .fit import FitConfig, Fitter, synthetic_init
from .mlp import TileMLP
from .scenes import multiplane_targets_device, rgb_crop_like_1080p

TILE = 16
SLOTS = 12
PER_SLOT = 13
IN_DIM = 4 * TILE * TILE
OUT_DIM = SLOTS * PER_SLOT
RAW_KEYS = ("means_2d", "pre_act_scales", "pre_act_rotation", "colours", "pre_act_phase", "pre_act_opacities",
            "curvature")


def tile_grid(H, W):
    return (H + TILE - 1) // TILE, (W + TILE - 1) // TILE


def num_gaussians(H, W):
    ty, tx = tile_grid(H, W)
    return ty * tx * SLOTS


def tile_features(image, depth, device="cuda"):
    """[tiles, 1024] float32: per tile RGB (768) then depth (256), tiles in row-major tile order."""
    img = torch.as_tensor(image, dtype=torch.float32, device=device)
    dep = torch.as_tensor(depth, dtype=torch.float32, device=device).reshape(1, *img.shape[1:])
    C, H, W = img.shape
    ty, tx = tile_grid(H, W)
    x = torch.zeros((C + 1, ty * TILE, tx * TILE), dtype=torch.float32, device=device)
    x[:C, :H, :W] = img
    x[C, :H, :W] = dep[0]
    x = x.view(C + 1, ty, TILE, tx, TILE).permute(1, 3, 0, 2, 4).reshape(ty * tx, (C + 1) * TILE * TILE)
    return x.contiguous()


def _slot_offsets():
    """Slot s starts at the centre of cell (s mod 4, s div 4) of a 4 x 3 grid over the tile (tile units)."""
    s = np.arange(SLOTS)
    return (s % 4 + 0.5) / 4.0, (s // 4 + 0.5) / 3.0


def grid_init(cfg: FitConfig, seed=0, jitter=0.05):
    """synthetic_init with the means stratified: 12 per tile on a jittered 4 x 3 grid."""
    H, W = cfg.H, cfg.W
    ty, tx = tile_grid(H, W)
    if cfg.num_gaussians != ty * tx * SLOTS:
        raise ValueError(f"grid_init needs num_gaussians = {ty * tx * SLOTS} (12 per 16x16 tile)")
    raw = synthetic_init(cfg, seed)
    rng = np.random.default_rng(seed + 7919)
    ou, ov = _slot_offsets()
    t = np.arange(ty * tx)
    x0 = (t % tx)[:, None] * TILE
    y0 = (t // tx)[:, None] * TILE
    mx = (x0 + TILE * (ou[None] + rng.uniform(-jitter, jitter, (len(t), SLOTS)))).ravel()
    my = (y0 + TILE * (ov[None] + rng.uniform(-jitter, jitter, (len(t), SLOTS)))).ravel()
    mx = np.clip(mx, 0.5, W - 0.5)
    my = np.clip(my, 0.5, H - 0.5)
    nm = np.stack([mx / W * 2 - 1, my / H * 2 - 1], 1)
    raw["means_2d"] = torch.from_numpy(np.arctanh(np.clip(nm, -0.999, 0.999)).astype(np.float32))
    return raw


def encode(raw, H, W):
    """Raw parameters of a grid-initialised fit -> regression targets [tiles, 156] (torch, raw's device)."""
    ty, tx = tile_grid(H, W)
    T = ty * tx
    m = raw["means_2d"].float().reshape(T, SLOTS, 2)
    mu_x = (torch.tanh(m[..., 0]) + 1) * 0.5 * W
    mu_y = (torch.tanh(m[..., 1]) + 1) * 0.5 * H
    t = torch.arange(T, device=m.device)
    u = (mu_x - ((t % tx) * TILE)[:, None].float()) / TILE
    v = (mu_y - ((t // tx) * TILE)[:, None].float()) / TILE
    sc = raw["pre_act_scales"].float().reshape(T, SLOTS, 2)
    rot = torch.remainder(raw["pre_act_rotation"].float().reshape(T, SLOTS, 1), math.pi)
    col = raw["colours"].float().reshape(T, SLOTS, 3)
    ph = torch.remainder(raw["pre_act_phase"].float().reshape(T, SLOTS, 3), 2 * math.pi)
    op = raw["pre_act_opacities"].float().reshape(T, SLOTS, 1)
    cv = raw["curvature"].float().reshape(T, SLOTS, 1)
    out = torch.cat([u[..., None], v[..., None], sc, rot, col, ph, op, cv], -1)
    return out.reshape(T, OUT_DIM).contiguous()


def decode(Y, H, W):
    """Predicted [tiles, 156] -> raw parameter dict (torch, Y's device), 12 Gaussians per tile."""
    ty, tx = tile_grid(H, W)
    T = ty * tx
    y = Y.float().reshape(T, SLOTS, PER_SLOT)
    t = torch.arange(T, device=y.device)
    mx = ((t % tx) * TILE)[:, None].float() + y[..., 0] * TILE
    my = ((t // tx) * TILE)[:, None].float() + y[..., 1] * TILE
    mx = mx.clamp(0.5, W - 0.5)
    my = my.clamp(0.5, H - 0.5)
    nm = torch.stack([mx / W * 2 - 1, my / H * 2 - 1], -1).clamp(-0.999, 0.999)
    return {"means_2d": torch.atanh(nm).reshape(-1, 2),
            "pre_act_scales": y[..., 2:4].reshape(-1, 2),
            "pre_act_rotation": y[..., 4].reshape(-1),
            "colours": y[..., 5:8].reshape(-1, 3),
            "pre_act_phase": y[..., 8:11].reshape(-1, 3),
            "pre_act_opacities": y[..., 11].reshape(-1),
            "curvature": y[..., 12].reshape(-1)}


def scene_config(H, W, iters, seed=0, **kw):
    """FitConfig of the headline RGB setting (639/515/473 nm, 3.74 um, 3 planes) at H x W, 12 Gaussians per tile."""
    base = dict(img_size=(W, H), num_gaussians=num_gaussians(H, W), wavelengths=[639e-9, 515e-9, 473e-9],
                pixel_pitch=3.74e-6, num_planes=3, d_val=1e-3, volume_depth=1e-3, num_itrs=iters, seed=seed,
                autotune=True)
    base.update(kw)
    return FitConfig(**base)


def make_scene(H, W, seed, device="cuda"):
    img, depth = rgb_crop_like_1080p(H, W, seed=seed)
    targets, q = multiplane_targets_device(img, depth, 3, device=device)
    return img, depth, targets, q


def make_pairs(num_scenes, H=256, W=256, iters=400, seed0=1000, slots=4, device="cuda", init_weights=None):
    """(X [n_tiles, 1024], T [n_tiles, 156]) from fits of seeded scenes run by the batched fitter.

    The fits start from ``grid_init`` or, when ``init_weights`` (a trained
    TileMLP weight vector) is given, from that network's prediction: a second
    round whose converged parameters stay close to a consistent start."""
    feats, jobs = {}, []
    for i in range(num_scenes):
        seed = seed0 + i
        img, depth, targets, q = make_scene(H, W, seed, device)
        cfg = scene_config(H, W, iters, seed=seed)
        feats[seed] = tile_features(img, depth, device)
        init = grid_init(cfg, seed) if init_weights is None else predict(init_weights, img, depth, device)
        jobs.append(FitJob(cfg, targets, q, iters, init=init, tag=seed))
    bf = BatchedFitter(jobs, slots=slots, device=device)
    results = bf.run()
    X = torch.cat([feats[r.tag] for r in results])
    T = torch.cat([encode(r.raw, H, W) for r in results])
    psnr = np.array([r.evaluation["psnr"] for r in results])
    return X, T, dict(fits=len(results), graph_launches=bf.graph_launches, mean_psnr=psnr.mean(0).tolist())


def constant_init(T, H, W, device="cuda"):
    """Ablation without the network: every slot at the mean training target of its kind
    (means on the slot grid), i.e. what an MLP that ignores its input would predict."""
    ty, tx = tile_grid(H, W)
    mean = T.reshape(-1, SLOTS, PER_SLOT).mean(0)
    return decode(mean.reshape(1, OUT_DIM).repeat(ty * tx, 1).to(device), H, W)


def output_weights(T):
    """Per-output loss weights: 1 / variance of each of the 13 parameter kinds over the training targets."""
    var = T.reshape(-1, SLOTS, PER_SLOT).var(dim=(0, 1)).clamp_min(1e-6)
    return (1.0 / var).repeat(SLOTS).float().contiguous()


def train(X, T, steps=2000, batch=8192, lr=3e-4, seed=0, log_every=0, val_fraction=0.1, val_every=0):
    """Fit a TileMLP to (X, T) with Adam on minibatches; returns (net, output weights, loss curve).

    The last `val_fraction` of the rows (whole scenes: make_pairs stacks them scene by scene) are held
    out. Every `val_every` steps (default steps / 20) the weighted validation loss is measured and the
    net keeps the weights of the best one (early stopping: longer training overfits the training
    scenes). The curve holds (step, train loss) pairs and, under "val", (step, validation loss)."""
    dev = X.device
    n_all = X.shape[0]
    n_val = int(n_all * val_fraction) if val_fraction > 0 else 0
    n = n_all - n_val
    batch = min(batch, n)
    net = TileMLP(batch, IN_DIM, 512, OUT_DIM, lr=lr, device=dev)
    wout = output_weights(T[:n])
    g = torch.Generator(device=dev).manual_seed(seed)
    xb = torch.empty((batch, IN_DIM), dtype=torch.float32, device=dev)
    tb = torch.empty((batch, OUT_DIM), dtype=torch.float32, device=dev)
    curve, val_curve = [], []
    if n_val > 0:
        val_every = val_every or max(1, steps // 20)
        chunk = min(batch, n_val)
        n_val -= n_val % chunk
        val_net = TileMLP(chunk, IN_DIM, 512, OUT_DIM, weights=net.weights, device=dev)  # shares net.weights
        best, best_loss = net.weights.clone(), float("inf")

    def validate():
        val_net.sync()
        tot = torch.zeros((), dtype=torch.float64, device=dev)
        for a in range(n, n + n_val, chunk):
            y = val_net.forward(X[a:a + chunk])
            tot += (((y - T[a:a + chunk]) ** 2) * wout).sum(dtype=torch.float64)
        return float(tot) / max(n_val, 1)

    for it in range(steps):
        idx = torch.randint(0, n, (batch,), generator=g, device=dev)
        torch.index_select(X, 0, idx, out=xb)
        torch.index_select(T, 0, idx, out=tb)
        loss = net.train_step(xb, tb, wout)
        if log_every and (it % log_every == 0 or it == steps - 1):
            curve.append((it, float(loss.item())))
        if n_val > 0 and ((it + 1) % val_every == 0 or it == steps - 1):
            v = validate()
            val_curve.append((it, v))
            if v < best_loss:
                best_loss = v
                best.copy_(net.weights)
    if n_val > 0:
        net.weights.copy_(best)
        net.sync()
        curve = dict(train=curve, val=val_curve, best_val=best_loss)
    return net, wout, curve


def predict(net_weights, image, depth, device="cuda"):
    """Raw parameters for a Fitter from the trained weights (any image size)."""
    X = tile_features(image, depth, device)
    net = TileMLP(X.shape[0], IN_DIM, 512, OUT_DIM, weights=net_weights, device=device)
    Y = net.forward(X)
    C, H, W = torch.as_tensor(image).shape
    return decode(Y, H, W)


def _timed_capture(fitter):
    """Fitter.capture() runs one iteration eagerly before recording the graph: its device time."""
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    fitter.capture()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / 1e3


def psnr_trace(fitter, iters, eval_every):
    """Run `iters` graph-replayed iterations; returns [(fit_seconds, iteration, per-plane PSNR)]."""
    trace = [(0.0, 0, fitter.evaluate()["psnr"])]
    spent = _timed_capture(fitter)  # the capture runs (and times) the first iteration
    done = 1
    while done < iters:
        n = min(eval_every, iters - done)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fitter.run(n)
        e.record()
        torch.cuda.synchronize()
        spent += s.elapsed_time(e) / 1e3
        done += n
        trace.append((spent, done, fitter.evaluate()["psnr"]))
    return trace


def time_to_psnr(trace, goal):
    """First fit time at which every plane's PSNR reaches the goal (None if never)."""
    for t, it, p in trace:
        if np.all(np.asarray(p) >= np.asarray(goal) - 1e-9):
            return t, it
    return None, None


def train_initialiser(num_scenes=64, H=256, W=256, iters=400, steps=3000, slots=4, device="cuda", seed0=1000):
    """Two-round training: fits from grid_init -> MLP 1; fits from MLP 1's prediction -> MLP 2.

    Returns (weights of MLP 2, round-2 targets (for the constant-init ablation), info)."""
    X, T, info1 = make_pairs(num_scenes, H, W, iters=iters, slots=slots, device=device, seed0=seed0)
    net1, _, c1 = train(X, T, steps=steps, lr=1e-3, log_every=max(1, steps // 4))
    X2, T2, info2 = make_pairs(num_scenes, H, W, iters=iters, slots=slots, device=device, seed0=seed0,
                               init_weights=net1.weights)
    net2, _, c2 = train(X2, T2, steps=steps, lr=1e-3, log_every=max(1, steps // 4))
    info = dict(round1=info1, round2=info2, loss_round1=c1, loss_round2=c2, pairs=int(X2.shape[0]))
    return net2.weights.detach().clone(), T2, info


def time_to_psnr_experiment(weights, T_ref, H=1080, W=1920, plain_iters=2000, eval_every=50, seed=0,
                            device="cuda", goal_every=10):
    """Plain (random) init vs learned init vs constant-mean init on one seeded H x W scene.

    The plain fit runs `plain_iters` iterations; its final per-plane PSNR is the
    goal. The other two run until every plane reaches the goal (at most
    `plain_iters`), checked every `goal_every` iterations. Times are fit-iteration
    time on the device (CUDA events, every iteration included, evaluations
    excluded), plus, for the learned init, the prediction itself."""
    img, depth, targets, q = make_scene(H, W, seed + 424242, device)
    out = {}
    cfg = scene_config(H, W, plain_iters, seed=seed)
    plain = Fitter(cfg, targets, q, init=synthetic_init(cfg, seed), device=device)
    tr = psnr_trace(plain, plain_iters, eval_every)
    goal = tr[-1][2]
    out["plain"] = dict(seconds=tr[-1][0], iters=plain_iters, psnr=np.round(goal, 3).tolist(),
                        psnr_start=np.round(tr[0][2], 3).tolist())
    del plain
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    init = predict(weights, img, depth, device)
    e.record()
    torch.cuda.synchronize()
    t_pred = s.elapsed_time(e) / 1e3
    for name, ini, extra in (("learned", init, t_pred), ("constant", constant_init(T_ref, H, W, device), 0.0)):
        cfg = scene_config(H, W, plain_iters, seed=seed)
        f = Fitter(cfg, targets, q, init={k: v.detach().cpu() for k, v in ini.items()}, device=device)
        p0 = f.evaluate()["psnr"]
        trace = []
        spent, done = _timed_capture(f), 1
        reached = None
        while done < plain_iters:
            n = min(goal_every, plain_iters - done)
            s.record()
            f.run(n)
            e.record()
            torch.cuda.synchronize()
            spent += s.elapsed_time(e) / 1e3
            done += n
            p = f.evaluate()["psnr"]
            trace.append((spent, done, p))
            if np.all(p >= goal):
                reached = (spent + extra, done)
                break
        out[name] = dict(seconds_to_goal=None if reached is None else reached[0],
                         iters_to_goal=None if reached is None else reached[1],
                         psnr_start=np.round(p0, 3).tolist(),
                         psnr_at_stop=np.round(trace[-1][2], 3).tolist(),
                         fraction_of_plain=None if reached is None else reached[0] / out["plain"]["seconds"])
        if name == "learned":
            out[name]["predict_seconds"] = t_pred
        del f
    out["goal_psnr"] = np.round(goal, 3).tolist()
    return out
