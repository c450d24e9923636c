"""Batched fitter: many fits of uneven size driven as one CUDA graph per iteration.

The reference fits one hologram per process (train_2d_gaussian_rgb.py). Here a
work queue of fit jobs (any mix of image sizes, Gaussian counts and iteration
budgets) is served by up to ``slots`` resident fits. One captured CUDA graph
advances every resident fit by one iteration: the capture forks one stream
branch per fit (each branch is that fit's fused iteration, cvqpg_fit_step), so
the small fits' kernels run side by side on the GPU and one graph launch costs
one host call for all of them. When a fit reaches its budget its slot is
harvested (final parameters, noise-free evaluation) and refilled from the
queue, and the graph is captured again. Jobs are taken longest-first (cost =
pixels x iterations), the classic LPT order for uneven work.

Multi-GPU: ``shard(jobs, rank, world)`` splits the queue by cost across ranks;
the fits are independent, so no collective is needed.
"""
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional

import torch

from . import _lib
from .fit import FitConfig, Fitter


@dataclass
class FitJob:
    cfg: FitConfig
    targets: Any
    depth_plane: Any
    iters: int
    init: Optional[Dict[str, Any]] = None
    tag: Any = None

    def __post_init__(self):
        if int(self.iters) < 1:
            raise ValueError(f"a fit job needs at least one iteration (got {self.iters})")

    def cost(self):
        return self.cfg.W * self.cfg.H * self.iters


@dataclass
class FitResult:
    tag: Any
    raw: Dict[str, torch.Tensor]
    evaluation: Dict[str, Any]
    iters: int
    overflowed: bool
    history_tail: List[Any] = field(default_factory=list)


def shard(jobs, rank, world):
    """Greedy cost balance of the job list over `world` ranks; returns this rank's jobs."""
    loads = [0] * world
    mine = []
    for j in sorted(jobs, key=lambda j: -j.cost()):
        r = min(range(world), key=lambda i: loads[i])
        loads[r] += j.cost()
        if r == rank:
            mine.append(j)
    return mine


class BatchedFitter:
    """``slots``: at most this many resident fits. ``pixel_budget`` (optional): admit a fit only
    while the resident fits' pixels stay within the budget (one fit is always admitted), so that
    small images run many at a time and large ones a few, with memory bounded by the budget."""

    def __init__(self, jobs: List[FitJob], slots: int = 4, device="cuda", chunk: int = 64,
                 pixel_budget: Optional[int] = None):
        self.queue = sorted(jobs, key=lambda j: -j.cost())
        self.slots = max(1, int(slots))
        self.pixel_budget = pixel_budget
        self.device = torch.device(device)
        self.chunk = max(1, int(chunk))
        self.active = []      # [job, fitter, remaining]
        self.results = []
        self.graph_launches = 0
        self._graph = None
        self._streams = [torch.cuda.Stream(self.device) for _ in range(self.slots)]

    def _fits_budget(self, job):
        if self.pixel_budget is None or not self.active:
            return True
        used = sum(j.cfg.W * j.cfg.H for j, _, _ in self.active)
        return used + job.cfg.W * job.cfg.H <= self.pixel_budget

    def _admit(self):
        while self.queue and len(self.active) < self.slots and self._fits_budget(self.queue[0]):
            job = self.queue.pop(0)
            cfg = job.cfg
            if cfg.num_itrs != job.iters:
                cfg.num_itrs = job.iters
            f = Fitter(cfg, job.targets, job.depth_plane, init=job.init, device=self.device)
            f.step()  # first iteration eagerly: lazy per-kernel set-up stays out of the capture
            self.active.append([job, f, job.iters - f.iteration_count()])
        self._graph = None

    def _capture(self):
        s0 = torch.cuda.Stream(self.device)
        s0.wait_stream(torch.cuda.current_stream(self.device))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s0):
            g.capture_begin()
            fork = torch.cuda.Event()
            fork.record(s0)
            statuses = []
            for i, (_, f, _) in enumerate(self.active):
                st = self._streams[i]
                st.wait_event(fork)
                statuses.append(f._step_call(st.cuda_stream))
            for i in range(len(self.active)):
                s0.wait_stream(self._streams[i])
            g.capture_end()
        torch.cuda.current_stream(self.device).wait_stream(s0)
        for st in statuses:
            _lib.check(st, "cvqpg_fit_step (batched capture)")
        self._graph = g

    def _harvest(self):
        keep = []
        for job, f, rem in self.active:
            if rem > 0:
                keep.append([job, f, rem])
                continue
            ev = f.evaluate()
            raw = {k: f.raw(k).detach().clone() for k in ("means_2d", "pre_act_scales", "pre_act_rotation",
                                                          "colours", "pre_act_phase", "pre_act_opacities",
                                                          "curvature")}
            self.results.append(FitResult(job.tag, raw, ev, f.iteration_count(), f.overflowed(),
                                          f.history_records(last=1)))
        changed = len(keep) != len(self.active)
        self.active = keep
        return changed

    def run(self):
        """Serve the whole queue; returns the FitResult list in completion order."""
        self._admit()
        while self.active:
            if self._graph is None:
                self._capture()
            n = min(self.chunk, min(rem for _, _, rem in self.active))
            for _ in range(n):
                self._graph.replay()
            self.graph_launches += n
            for a in self.active:
                job, f = a[0], a[1]
                if f.overflowed():
                    # the overflowed steps changed nothing: grow the fit's pair capacity and
                    # let it run the missing iterations
                    f.grow_pair_capacity()
                    self._graph = None
                a[2] = job.iters - f.iteration_count()
            if self._harvest():
                self._graph = None  # the active set changed: capture again
                self._admit()
        torch.cuda.synchronize(self.device)
        return self.results
