"""The fused CVQPG fit loop on the B200 kernels.

``Fitter`` runs the reference training-loop body (train_2d_gaussian_rgb.py:179-211):

    render (preprocess, tile binning, splat) -> soft_window_pad + amplitude clamp
    -> BLASM to every plane -> multi-plane loss + SSIM -> backward
    -> nan_to_num -> clip_grad_norm_(1.0) -> Adan (per-group lrs, means cosine
    schedule, curvature warm-up)

as one call of ``cvqpg_fit_step`` per iteration, optionally captured once in a
CUDA graph and replayed. Parameters live in one flat device buffer whose
slices are exposed with the reference names and shapes (``means_2d``,
``pre_act_scales``, ... , model_2d_gaussian_rgb.py:18-26), and checkpoints use
the reference's ``save_gaussians`` keys (model_2d_gaussian_rgb.py:155-167).
"""
import ctypes
import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import torch

from . import _lib
from .loss import TARGET_RANGE_WORKSPACE_PER_PLANE
from .propagator import reference_distances, reference_pad_size

CULL_CUDA16_5SIGMA = 0
CULL_TORCH64_3SIGMA = 1
CULL_NONE = 2
CURV_MODES = {"off": 0, "constant": 1, "scale_aware": 2}
RAW_KEYS = ("means_2d", "pre_act_scales", "pre_act_rotation", "colours", "pre_act_phase", "pre_act_opacities",
            "curvature")


class FitParams(ctypes.Structure):
    _fields_ = [("channels", ctypes.c_int), ("planes", ctypes.c_int), ("height", ctypes.c_int),
                ("width", ctypes.c_int), ("pad_height", ctypes.c_int), ("pad_width", ctypes.c_int),
                ("num_gaussians", ctypes.c_int), ("pair_capacity", ctypes.c_int), ("cull_mode", ctypes.c_int),
                ("curv_mode", ctypes.c_int), ("curv_trainable", ctypes.c_int), ("warmup_iters", ctypes.c_int),
                ("num_iters", ctypes.c_int), ("history_len", ctypes.c_int), ("no_prox", ctypes.c_int),
                ("inject_noise", ctypes.c_int), ("pixel_pitch", ctypes.c_double),
                ("wavelengths", ctypes.c_double * 3), ("distances", ctypes.c_double * 8),
                ("aperture_radius", ctypes.c_double), ("curv_nyquist", ctypes.c_double),
                ("curv_const", ctypes.c_double), ("lr", ctypes.c_double * 6), ("betas", ctypes.c_double * 3),
                ("eps", ctypes.c_double), ("weight_decay", ctypes.c_double), ("max_grad_norm", ctypes.c_double),
                ("loss_weights", ctypes.c_float * 3), ("ssim_weight", ctypes.c_float),
                ("noise_ratio", ctypes.c_float), ("plan_hint", ctypes.c_int), ("seed", ctypes.c_ulonglong),
                ("target_moments", ctypes.c_void_p)]


@dataclass
class FitConfig:
    """Fit settings with the reference flag names (train_2d_gaussian_rgb.py:275-324)."""
    img_size: tuple = (640, 480)             # (W, H)
    num_gaussians: int = 30720
    wavelengths: List[float] = field(default_factory=lambda: [639e-9, 532e-9, 473e-9])
    pixel_pitch: float = 3.74e-6
    num_planes: int = 2
    d_val: float = 3e-3
    volume_depth: float = 4e-3
    pad_size: Optional[List[int]] = None     # [pH, pW]; default guard band of 144 px rounded to 64
    aperture_size: int = 0                   # 0 = disabled (10 * max(img_size)), -1 = sum/1.4, >0 radius
    primitive: str = "curv"                  # 'flat' or 'curv'
    curv_mode: str = "scale_aware"
    curv_nyquist: float = 0.9
    warmup_iters: int = 400
    num_itrs: int = 2001
    lr: float = 0.01                         # means lr; the other groups use the reference constants
    group_lrs: Optional[List[float]] = None  # override all 6 group lrs (means, scales, amp/phase, opac, rot, curv)
    cosine_means: bool = True                # MeansCosineScheduler (train_2d_gaussian_rgb.py:58-70)
    split_ratio: float = 1.0
    seed: int = 0
    cull: int = CULL_CUDA16_5SIGMA
    phase_iso: bool = False                  # isotropic quadratic phase (--phase_iso, model_2d_gaussian_rgb.py:356-359)
    pair_capacity: Optional[int] = None
    inject_noise: bool = True
    max_grad_norm: float = 1.0               # clip_grad_norm_ max_norm (train_2d_gaussian_rgb.py:209); <= 0: no clip
    history_len: int = 4096
    plan_hint: int = 0                       # FFT plan of the propagation (autotune.py); 0 = defaults
    autotune: bool = False                   # pick plan_hint by measurement (cached per grid)
    target_moments: bool = True              # precompute the targets' SSIM window moments once per fit

    @property
    def W(self):
        return int(self.img_size[0])

    @property
    def H(self):
        return int(self.img_size[1])

    def resolved_pad(self):
        return list(self.pad_size) if self.pad_size is not None else reference_pad_size(self.img_size)

    def resolved_aperture(self):
        if self.aperture_size < 0:
            return int(sum(self.img_size) / 1.4)
        if self.aperture_size == 0:
            return 10 * max(self.img_size)
        return self.aperture_size

    def distances(self):
        return reference_distances(self.num_planes, self.volume_depth, self.d_val)

    def lrs(self):
        if self.group_lrs is not None:
            return list(self.group_lrs)
        return [self.lr, 0.005, 0.0025, 0.025, 0.001, 0.001]  # train_2d_gaussian_rgb.py:75-82


def means_lr_table(base_lr, num_itrs, eta_min=1e-3):
    """Per-iteration means lr exactly as MeansCosineScheduler produces it (torch CosineAnnealingLR)."""
    p = torch.nn.Parameter(torch.zeros(1))
    opt = torch.optim.SGD([p], lr=base_lr)
    sch = torch.optim.lr_scheduler.CosineAnnealingLR(opt, T_max=max(1, num_itrs), eta_min=eta_min)
    out = []
    for _ in range(max(1, num_itrs)):
        out.append(opt.param_groups[0]["lr"])
        opt.step()
        sch.step()
    return np.array(out, dtype=np.float64)


def reference_init(cfg, generator=None):
    """Raw parameters as Gaussians2D._initialize_2d draws them (model_2d_gaussian_rgb.py:41-77)."""
    N, W, H, C = cfg.num_gaussians, cfg.W, cfg.H, len(cfg.wavelengths)
    g = generator
    m = torch.rand((N, 2), generator=g)
    m[:, 0] *= W
    m[:, 1] *= H
    nm = m.clone()
    nm[:, 0] = nm[:, 0] / W * 2 - 1
    nm[:, 1] = nm[:, 1] / H * 2 - 1
    out = {"means_2d": torch.atanh(torch.clamp(nm, -0.999, 0.999))}
    out["colours"] = torch.rand((N, C), generator=g)
    out["pre_act_scales"] = torch.log(torch.rand((N, 2), generator=g) * 3.5 + 1.5)
    out["pre_act_rotation"] = torch.rand((N,), generator=g) * 2 * np.pi - np.pi
    out["pre_act_phase"] = torch.zeros((N, C))
    out["pre_act_opacities"] = torch.zeros((N,)) - 0.5
    out["curvature"] = torch.zeros((N,))
    return out


def synthetic_init(cfg, seed=0):
    """Raw parameters from the benchmark distributions: mu ~ U(image), log-scale ~ N(log 2 px, 0.3),
    rotation ~ U(0, pi), amplitude ~ U(0, 1), phase ~ U(0, 2 pi), kappa ~ N(0, 0.01 rad/px^2) where
    kappa = k_min * c * |sx sy| * dxy^2 / 2 is the quadratic-phase coefficient on the Mahalanobis
    distance, inverted through the scale-aware curvature bound (model_2d_gaussian_rgb.py:95-107)."""
    rng = np.random.default_rng(seed)
    N, W, H, C = cfg.num_gaussians, cfg.W, cfg.H, len(cfg.wavelengths)
    mx, my = rng.uniform(0, W, N), rng.uniform(0, H, N)
    means = np.arctanh(np.clip(np.stack([mx / W * 2 - 1, my / H * 2 - 1], 1), -0.999, 0.999))
    s = np.exp(rng.normal(math.log(2.0), 0.3, (N, 2)))
    scales = np.log(np.maximum(s - 0.1, 1e-3))   # activation adds 0.1
    rot = rng.uniform(0, math.pi, N)
    col = rng.uniform(0, 1, (N, C))
    ph = rng.uniform(0, 2 * math.pi, (N, C))
    opac = np.full(N, -0.5)
    lam = min(cfg.wavelengths) if C == 3 else cfg.wavelengths[0]
    kmin = 2 * math.pi / lam
    dxy2 = cfg.pixel_pitch ** 2
    kappa = rng.normal(0, 0.01, N)
    c = 2 * kappa / (kmin * s[:, 0] * s[:, 1] * dxy2)
    cmax = cfg.curv_nyquist * lam / (6.0 * s.max(1) * dxy2)
    curv = np.arctanh(np.clip(c / cmax, -0.999, 0.999))
    arr = dict(means_2d=means, pre_act_scales=scales, pre_act_rotation=rot, colours=col, pre_act_phase=ph,
               pre_act_opacities=opac, curvature=curv)
    return {k: torch.from_numpy(np.asarray(v, dtype=np.float32)) for k, v in arr.items()}



def compute_target_moments(p, targets, out=None):
    """Windowed SSIM moments of fixed targets (cvqpg_loss_target_moments) for a fit's loss,
    into `out` when given."""
    from .loss import LossParams
    lib = _lib.lib()
    P, C, H, W = p.planes, p.channels, p.height, p.width
    lp = LossParams(C, P, H, W, 1.0, 1.0, 1.0, 0.0, 0.0, 0, 0)
    nbytes = _lib.size_query(lib.cvqpg_loss_target_moments_size, ctypes.byref(lp))
    mom = out if out is not None else torch.empty(nbytes // 4, dtype=torch.float32, device=targets.device)
    if mom.numel() * 4 < nbytes:
        raise ValueError("target moments buffer too small")
    _lib.check(lib.cvqpg_loss_target_moments(ctypes.byref(lp), _lib.ptr(targets), _lib.ptr(mom), nbytes,
                                             _lib.stream_of(targets.device)), "cvqpg_loss_target_moments")
    return mom

def save_gaussians(raw, img_size, path):
    """Write a checkpoint in the reference's format (Gaussians2D.save_gaussians,
    model_2d_gaussian_rgb.py:155-167): the seven raw tensors as CPU float32 tensors and img_size,
    under the reference's keys, so that Gaussians2D.load_gaussians and export_poh.py read it."""
    d = {k: torch.as_tensor(raw[k], dtype=torch.float32).detach().cpu().clone() for k in RAW_KEYS}
    d["img_size"] = tuple(int(v) for v in img_size)
    torch.save(d, path)
    return d


def read_gaussians(path):
    """Read a reference-format checkpoint: ({raw key: float32 tensor}, img_size)."""
    d = torch.load(path, map_location="cpu")
    missing = [k for k in RAW_KEYS if k not in d]
    if missing:
        raise ValueError(f"checkpoint {path} lacks {missing}")
    return {k: d[k].detach().to(torch.float32) for k in RAW_KEYS}, tuple(int(v) for v in d.get("img_size", (0, 0)))


class Fitter:
    """Device-resident fit of one hologram with the fused kernels."""

    def __init__(self, cfg: FitConfig, targets, depth_plane, init=None, device="cuda"):
        self.cfg = cfg
        self.device = torch.device(device)
        C, P, H, W, N = len(cfg.wavelengths), cfg.num_planes, cfg.H, cfg.W, cfg.num_gaussians
        if C not in (1, 3):
            raise ValueError("1 or 3 wavelengths")
        if P > 8:
            raise ValueError("at most 8 planes")
        self.C, self.P, self.H, self.W, self.N = C, P, H, W, N
        p = FitParams()
        pad = cfg.resolved_pad()
        p.channels, p.planes, p.height, p.width = C, P, H, W
        p.pad_height, p.pad_width = int(pad[0]), int(pad[1])
        p.num_gaussians = N
        p.pair_capacity = int(cfg.pair_capacity if cfg.pair_capacity else max(1 << 16, 24 * N))
        p.cull_mode = int(cfg.cull) | (0x100 if cfg.phase_iso else 0)  # CVQPG_PHASE_ISO
        flat = cfg.primitive == "flat"
        p.curv_mode = 0 if flat else CURV_MODES[cfg.curv_mode]
        p.curv_trainable = 0 if flat else 1
        p.warmup_iters = 0 if flat else int(cfg.warmup_iters)
        p.num_iters = max(1, int(cfg.num_itrs))
        p.history_len = int(cfg.history_len)
        p.no_prox = 0
        p.inject_noise = 1 if cfg.inject_noise else 0
        p.pixel_pitch = float(cfg.pixel_pitch)
        for i, wl in enumerate(cfg.wavelengths):
            p.wavelengths[i] = float(wl)
        for i, z in enumerate(cfg.distances()):
            p.distances[i] = float(z)
        p.aperture_radius = float(cfg.resolved_aperture())
        p.curv_nyquist = float(cfg.curv_nyquist)
        p.curv_const = 200.0
        for i, lr in enumerate(cfg.lrs()):
            p.lr[i] = float(lr)
        for i, b in enumerate((0.98, 0.92, 0.99)):
            p.betas[i] = b
        p.eps, p.weight_decay, p.max_grad_norm = 1e-8, 0.0, float(cfg.max_grad_norm)
        for i in range(3):
            p.loss_weights[i] = 1.0
        p.ssim_weight = 0.025 * 0.2
        p.noise_ratio = 1e-3
        p.seed = int(cfg.seed)
        p.plan_hint = int(cfg.plan_hint)
        if cfg.autotune:
            from .autotune import tune_for
            p.plan_hint = int(tune_for(cfg, device=device)[0])
        self.plan_hint = p.plan_hint
        self.params = p
        lib = _lib.lib()
        self._lib = lib
        total = (7 + 2 * C) * N
        self.numels = [2 * N, 2 * N, N, C * N, C * N, N, N]
        self.shapes = [(N, 2), (N, 2), (N,), (N, C), (N, C), (N,), (N,)]
        self._lr_table = means_lr_table(cfg.lr, p.num_iters) if cfg.cosine_means else None
        with torch.cuda.device(self.device):
            self._setup_workspace()
            self.flat = torch.zeros(total, dtype=torch.float32, device=self.device)
            self.grads = torch.zeros(total, dtype=torch.float32, device=self.device)
            self.adan_state = torch.zeros(4 * total, dtype=torch.float32, device=self.device)
            self.iteration = torch.zeros(1, dtype=torch.int32, device=self.device)
            self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
            self.history = torch.zeros(p.history_len, 1 + 3 * P, dtype=torch.float32, device=self.device)
            self.targets = torch.as_tensor(targets, dtype=torch.float32).to(self.device).contiguous()
            self.depth_plane = torch.as_tensor(depth_plane).to(torch.uint8).to(self.device).contiguous()
            if tuple(self.targets.shape) != (P, C, H, W) or tuple(self.depth_plane.shape) != (H, W):
                raise ValueError("targets must be [P,C,H,W] and depth_plane [H,W]")
            self.target_range = torch.empty(P, dtype=torch.float32, device=self.device)
            self._range_scratch = _lib.workspace(P * TARGET_RANGE_WORKSPACE_PER_PLANE, self.device)
            self.target_moments = None
            if cfg.target_moments:
                self.target_moments = compute_target_moments(p, self.targets)
                p.target_moments = _lib.ptr(self.target_moments)
            self.refresh_targets()
        if init is None:
            init = synthetic_init(cfg, cfg.seed)
        self.load_raw(init)
        self._graph = None
        self._issued = 0        # steps issued through run()/capture (host count)
        self._since_check = 0   # steps issued since the status was last read
        self._eval_out = torch.zeros(1 + 3 * P, dtype=torch.float32, device=self.device)

    def _setup_workspace(self):
        """(Re)carve the workspace for the current params (pair capacity included) and fill its tables."""
        p, lib = self.params, self._lib
        self.ws_bytes = _lib.size_query(lib.cvqpg_fit_workspace_size, ctypes.byref(p))
        self.workspace = None
        self.workspace = torch.empty(self.ws_bytes, dtype=torch.uint8, device=self.device)
        table = self._lr_table
        tptr = table.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if table is not None else None
        _lib.check(lib.cvqpg_fit_setup(ctypes.byref(p), tptr, _lib.ptr(self.workspace), self.ws_bytes),
                   "cvqpg_fit_setup")

    def pair_count(self):
        """(true tile-pair total, overflowed) of the last step or evaluation (host read)."""
        out = torch.zeros(2, dtype=torch.int32, device=self.device)
        _lib.check(self._lib.cvqpg_fit_pair_count(ctypes.byref(self.params), _lib.ptr(self.workspace),
                                                  self.ws_bytes, _lib.ptr(out), _lib.stream_of(self.device)),
                   "cvqpg_fit_pair_count")
        a = out.cpu().tolist()
        return int(a[0]), bool(a[1])

    def grow_pair_capacity(self, needed=None):
        """Enlarge the tile-pair capacity after an overflow: to 1.25x the pair total of the last
        step (at least double the old capacity), with a new workspace; clears the status flag and
        drops the captured graph. The overflowed step changed nothing, so the fit resumes at the
        same iteration."""
        if needed is None:
            needed, _ = self.pair_count()
        old = int(self.params.pair_capacity)
        new = max(2 * old, int(1.25 * needed) + 1024)
        if new >= 2 ** 31 - 1:
            raise RuntimeError(f"tile pairs ({needed}) exceed the int32 capacity of the binning")
        self.params.pair_capacity = new
        with torch.cuda.device(self.device):
            self._setup_workspace()
        self.status.bitwise_and_(~1)
        self._graph = None
        self.capacity_grown = getattr(self, "capacity_grown", 0) + 1
        return new

    def refresh_targets(self):
        """Recompute what the loss derives from `targets` (the per-plane range of the noise and the
        SSIM window moments) into the same buffers, so a captured graph stays valid. Call it after
        changing `targets` in place."""
        P, C, H, W = self.P, self.C, self.H, self.W
        lib, dev = self._lib, self.device
        _lib.check(lib.cvqpg_loss_target_range(_lib.ptr(self.targets), P, C, H, W, _lib.ptr(self.target_range),
                                               _lib.ptr(self._range_scratch), self._range_scratch.numel(),
                                               _lib.stream_of(dev)), "cvqpg_loss_target_range")
        if self.target_moments is not None:
            compute_target_moments(self.params, self.targets, out=self.target_moments)

    # -- parameters ------------------------------------------------------------------------
    def grad(self, name):
        """Gradient of raw parameter `name` from the last step (after nan_to_num and the clip)."""
        i = RAW_KEYS.index(name)
        off = sum(self.numels[:i])
        return self.grads[off:off + self.numels[i]].view(self.shapes[i])

    def raw(self, name):
        i = RAW_KEYS.index(name)
        off = sum(self.numels[:i])
        return self.flat[off:off + self.numels[i]].view(self.shapes[i])

    def load_raw(self, raw):
        for k in RAW_KEYS:
            self.raw(k).copy_(torch.as_tensor(raw[k], dtype=torch.float32).reshape(self.raw(k).shape))

    def state_dict(self):
        """Reference checkpoint keys (model_2d_gaussian_rgb.py:155-167)."""
        d = {k: self.raw(k).detach().cpu().clone() for k in RAW_KEYS}
        d["img_size"] = tuple(self.cfg.img_size)
        return d

    def save_gaussians(self, path):
        save_gaussians({k: self.raw(k) for k in RAW_KEYS}, self.cfg.img_size, path)

    def reset_optimizer(self):
        """Fresh Adan state, iteration 0 and an empty history (the reference builds a new optimiser
        after loading, train_2d_gaussian_rgb.py:73-86)."""
        self.adan_state.zero_()
        self.grads.zero_()
        self.iteration.zero_()
        self.history.zero_()
        self.status.zero_()
        self._issued = 0
        self._since_check = 0

    def load_gaussians(self, path):
        """Load a reference-format checkpoint (model_2d_gaussian_rgb.py:170-180) into this fit: the
        image size must match; the optimiser state, iteration counter and history start afresh."""
        d, size = read_gaussians(path)
        if size != (self.cfg.W, self.cfg.H):
            raise ValueError(f"checkpoint img_size {size} does not match the fit's {(self.cfg.W, self.cfg.H)}")
        for k in RAW_KEYS:
            if d[k].numel() != self.raw(k).numel():
                raise ValueError(f"checkpoint {k} has {d[k].numel()} values, the fit expects {self.raw(k).numel()}")
        self.load_raw(d)
        self.reset_optimizer()

    # -- iteration -------------------------------------------------------------------------
    def _step_call(self, stream):
        p = self.params
        return self._lib.cvqpg_fit_step(
            ctypes.byref(p), _lib.ptr(self.flat), _lib.ptr(self.grads), _lib.ptr(self.adan_state),
            _lib.ptr(self.targets), _lib.ptr(self.depth_plane), _lib.ptr(self.target_range), _lib.ptr(self.iteration),
            _lib.ptr(self.history), _lib.ptr(self.status), _lib.ptr(self.workspace), self.ws_bytes,
            ctypes.c_void_p(stream))

    STAGES = ("preprocess", "binning", "splat", "blasm_rows", "blasm_columns", "blasm_inverse_rows", "loss",
              "adjoint_rows", "adjoint_columns", "adjoint_inverse_rows", "splat_adjoint", "preprocess_adjoint",
              "clip_adan")

    def step_timed(self):
        """One eager iteration with CUDA events at the stage boundaries; returns {stage: ms} after a sync."""
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(len(self.STAGES) + 1)]
        s = torch.cuda.current_stream(self.device)
        for e in evs:  # materialise the event handles
            e.record(s)
        arr = (ctypes.c_void_p * len(evs))(*[ctypes.c_void_p(e.cuda_event) for e in evs])
        p = self.params
        st = self._lib.cvqpg_fit_step_timed(
            ctypes.byref(p), _lib.ptr(self.flat), _lib.ptr(self.grads), _lib.ptr(self.adan_state),
            _lib.ptr(self.targets), _lib.ptr(self.depth_plane), _lib.ptr(self.target_range), _lib.ptr(self.iteration),
            _lib.ptr(self.history), _lib.ptr(self.status), _lib.ptr(self.workspace), self.ws_bytes,
            ctypes.c_void_p(s.cuda_stream), arr, len(evs))
        _lib.check(st, "cvqpg_fit_step_timed")
        torch.cuda.synchronize(self.device)
        return {name: evs[i].elapsed_time(evs[i + 1]) for i, name in enumerate(self.STAGES)}

    def step(self):
        """One fit iteration (eager launches on the current stream). A step whose tile pairs
        overflow changes nothing and sets overflowed(); run() and check_status() recover from it."""
        s = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._step_call(s), "cvqpg_fit_step")
        self._issued += 1
        self._since_check += 1

    def capture(self):
        """Record one iteration into a CUDA graph (the iteration state is in device memory)."""
        self.step()  # warm kernels / lazy attribute setup outside capture
        torch.cuda.synchronize(self.device)
        try:
            g = torch.cuda.CUDAGraph(keep_graph=True)  # keep the cudaGraph_t for node inspection
        except TypeError:
            g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            g.capture_begin()
            st = self._step_call(s.cuda_stream)
            g.capture_end()
        torch.cuda.current_stream(self.device).wait_stream(s)
        _lib.check(st, "cvqpg_fit_step (capture)")
        self._graph = g
        return g

    def run(self, iters, graph=True, check_every=100):
        """Advance the fit by `iters` iterations (graph replays, or eager steps). Every
        `check_every` iterations, counted across calls, the status flag is read (one host sync):
        if a step's tile pairs overflowed the capacity, that step changed nothing, so the capacity
        is grown (grow_pair_capacity) and the lost iterations run again. check_status() does the
        same check on demand (for the last iterations of a fit)."""
        left = max(0, int(iters))
        while left > 0:
            n = min(left, max(1, int(check_every) - self._since_check))
            left -= n
            if graph and self._graph is None:
                self.capture()  # runs (and counts) one step itself
                n -= 1
            if graph:
                for _ in range(n):
                    self._graph.replay()
                self._issued += n
                self._since_check += n
            else:
                for _ in range(n):
                    self.step()
            if self._since_check >= max(1, int(check_every)):
                left += self._recover_overflow()

    def check_status(self):
        """Read the status flag now; after an overflow, grow the capacity and run the lost iterations
        again. Returns the number of iterations that were run again."""
        lost = self._recover_overflow()
        if lost:
            self.run(lost)
            self._recover_overflow()
        return lost

    def _recover_overflow(self):
        self._since_check = 0
        if not self.overflowed():
            return 0
        done = self.iteration_count()
        lost = max(0, self._issued - done)
        self._issued = done
        self.grow_pair_capacity()
        return lost

    def evaluate(self, field_out=None, planes_out=None):
        """Noise-free forward at the current parameters: dict of loss, per-plane MSE/PSNR/SSIM."""
        p = self.params
        st = self._lib.cvqpg_fit_evaluate(
            ctypes.byref(p), _lib.ptr(self.flat), _lib.ptr(self.targets), _lib.ptr(self.depth_plane),
            _lib.ptr(self.target_range), _lib.ptr(self._eval_out),
            _lib.ptr(torch.view_as_real(field_out)) if field_out is not None else None,
            _lib.ptr(torch.view_as_real(planes_out)) if planes_out is not None else None, _lib.ptr(self.status),
            _lib.ptr(self.workspace), self.ws_bytes, _lib.stream_of(self.device))
        _lib.check(st, "cvqpg_fit_evaluate")
        o = self._eval_out.cpu().numpy().astype(np.float64)
        P = self.P
        mse = o[1:1 + P]
        return dict(loss=float(o[0]), mse=mse, psnr=-10.0 * np.log10(np.maximum(mse, 1e-30)),
                    ssim=o[1 + P:1 + 2 * P], plane_loss=o[1 + 2 * P:1 + 3 * P])

    def iteration_count(self):
        return int(self.iteration.item())

    def overflowed(self):
        """A step's tile pairs exceeded the capacity (status bit 0)."""
        return bool(int(self.status.item()) & 1)

    def nonfinite(self):
        """A step's loss was NaN or Inf (status bit 1)."""
        return bool(int(self.status.item()) & 2)

    def history_records(self, last=None):
        """(iteration, loss, mse[P], ssim[P]) for the recorded iterations (host read)."""
        it = self.iteration_count()
        h = self.history.cpu().numpy()
        n = min(it, h.shape[0]) if last is None else min(last, it, h.shape[0])
        rows = [(i, h[i % h.shape[0]]) for i in range(it - n, it)]
        P = self.P
        return [(i, float(r[0]), r[1:1 + P].copy(), r[1 + P:1 + 2 * P].copy()) for i, r in rows]
