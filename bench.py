#!/usr/bin/env python
"""Benchmark: CVQPG hologram-fit iterations per second on B200.

Workload (default ``rgb1080``): 1920x1080 RGB (639/515/473 nm, 3.74 um pitch),
96,000 curvature Gaussians, BLASM to 3 planes at 0.5/1.0/1.5 mm (pad
1408x2240, FFT grid 2816x4480), seeded synthetic target (2,000 coloured
anisotropic blobs + 1/f noise) and 1/f depth; one step = one full fit
iteration (render, propagate, multi-plane loss + SSIM, backward, clip, Adan).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference|reference-gpu]

``--impl ours`` (default): the fused sm_100a iteration replayed from a CUDA
graph; prints one JSON line with value (it/s over all ranks), the roofline of
the dominant HBM-bound kernel, e2e through the public Fitter API with pinned
host buffers, the CPU baseline, clocks and the kernel-launch count.
``--impl reference``: the reference's CPU implementation (the oracle's torch
port of the reference fit loop) on the host cores, every step a bounded
sample of one iteration's components (see ``cpu_sample_step``).
``--impl reference-gpu``: the reference's own CUDA rasterizer (compiled from
its sources into oracle/_ref) with the torch/cuFFT propagator, loss and Adan of
the reference loop, on the same GPU.
Multi-GPU: a single fit does not shard; N ranks run N independent replicas
(different seeds) and value = total iterations / max elapsed over ranks.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = "1080p RGB fit iters/sec; time-to-plain-PSNR, learned vs plain init, 1×B200"
WORKLOADS = {
    "rgb1080": dict(W=1920, H=1080, N=96000, P=3, wl=[639e-9, 515e-9, 473e-9], pitch=3.74e-6, d_val=1e-3,
                    vd=1e-3),
    "gray256": dict(W=256, H=256, N=4096, P=3, wl=[515e-9], pitch=8e-6, d_val=1.5e-3, vd=1e-3),
}


# ----------------------------------------------------------------------------------------------
# helpers
# ----------------------------------------------------------------------------------------------
def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def init_dist(world, local):
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        return dist
    return None


def barrier(dist):
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()


def max_over_ranks(dist, x):
    if dist is None:
        return x
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled in the background during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _sample(self):
        try:
            out = subprocess.run(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                  "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=10)
            if out.returncode == 0 and out.stdout.strip():
                self.rows.append([c.strip() for c in out.stdout.strip().split(",")])
        except Exception:
            pass

    def _run(self):
        while not self._stop.is_set():
            self._sample()
            self._stop.wait(0.1)

    def start(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=15)
        if not self.rows:
            self._sample()
        return self.summary()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        smax = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 4 + i and r[4 + i] == "Active"})
        pw = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(self.rows), "power_w_max": max(pw) if pw else None}


def device_smi_index(dev):
    try:
        p = torch.cuda.get_device_properties(dev)
        bus = getattr(p, "pci_bus_id", None)
        dom = getattr(p, "pci_domain_id", 0)
        devid = getattr(p, "pci_device_id", 0)
        if bus is not None:
            return f"{dom:08X}:{bus:02X}:{devid:02X}.0"
    except Exception:
        pass
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        return vis.split(",")[dev]
    return str(dev)


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(stage, workload="rgb1080"):
    """DRAM bytes per launch of a stage from a committed ncu summary (profiles/*_<workload>.md), or
    None: the summaries hold captures of one workload, and another workload's launch moves other bytes."""
    pdir = os.path.join(REPO, "profiles")
    if not os.path.isdir(pdir):
        return None
    for name in sorted(os.listdir(pdir)):
        if not name.endswith(f"_{workload}.md"):
            continue
        with open(os.path.join(pdir, name)) as f:
            for line in f:
                if line.startswith(f"traffic_bytes_per_launch[{stage}]:"):
                    try:
                        return float(line.split(":", 1)[1].split()[0])
                    except ValueError:
                        return None
    return None


def count_graph_kernels(graph):
    """Kernel nodes in a captured torch CUDA graph (cuda-python), or None."""
    try:
        from cuda.bindings import runtime as rt
        g = rt.cudaGraph_t(init_value=graph.raw_cuda_graph())
        err, _, n = rt.cudaGraphGetNodes(g, 0)
        err, nodes, n = rt.cudaGraphGetNodes(g, n)
        kernels = 0
        for node in nodes:
            err, t = rt.cudaGraphNodeGetType(node)
            if t == rt.cudaGraphNodeType.cudaGraphNodeTypeKernel:
                kernels += 1
        return kernels
    except Exception:
        return None


def kernels_per_fit_step(cfg):
    """Kernel launches issued by one cvqpg_fit_step (from its launch sequence; memsets excluded)."""
    lists = ((cfg.W + 15) // 16) * ((cfg.H + 15) // 16)
    bits = max(1, math.ceil(math.log2(max(lists, 2))))
    passes = 1 if bits <= 8 else (bits + 7) // 8
    binning = 1 + 3 + 1 + 4 * passes + 1 + 1  # ... + ranges + tile order
    return 1 + binning + 1 + 3 + 2 + 1 + 3 + 1 + 1 + 2 + 1  # ... preprocess adjoint, Adan scalars + step, record


DATA = "synthetic (seeded blobs + 1/f noise targets, 1/f depth; random-init Gaussians)"


def workload_config(args, cfg, world):
    """The `config` object of every arm's JSON line (same keys for ours and the reference)."""
    pH, pW = cfg.resolved_pad()
    return {"workload": f"{args.workload}_fit", "image": f"{cfg.W}x{cfg.H}", "channels": len(cfg.wavelengths),
            "gaussians": cfg.num_gaussians, "planes": cfg.num_planes, "pad": f"{pH}x{pW}",
            "fft_grid": f"{2 * pH}x{2 * pW}", "primitive": args.primitive, "cull": "cuda16_5sigma",
            "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (per-iteration working set ~GBs)"}


def build_scene(wl, seed, device, ours=False):
    """Seeded scene and its multi-plane targets: with this library's target kernel for our arm,
    with the torch restatement of the reference's target synthesis for the reference arms."""
    from complex_valued_quadratic_phase_gaussian_b200 import scenes
    if len(wl["wl"]) == 3:
        img, depth = scenes.rgb_blobs(wl["H"], wl["W"], seed=seed)
    else:
        img, depth = scenes.grayscale_blobs(wl["H"], wl["W"], seed=seed)
    if ours:
        targets, q = scenes.multiplane_targets_device(img, depth, wl["P"], device=device)
    else:
        targets, q = scenes.multiplane_targets(img, depth, wl["P"], device=device)
    return img, depth, targets, q


def fit_config(wl, seed, primitive="curv"):
    from complex_valued_quadratic_phase_gaussian_b200.fit import FitConfig
    return FitConfig(img_size=(wl["W"], wl["H"]), num_gaussians=wl["N"], wavelengths=list(wl["wl"]),
                     pixel_pitch=wl["pitch"], num_planes=wl["P"], d_val=wl["d_val"], volume_depth=wl["vd"],
                     primitive=primitive, warmup_iters=400, num_itrs=2000, seed=seed, autotune=True)


def stage_bytes(cfg):
    """Algorithmic (compulsory) HBM bytes per launch of each BLASM/loss stage, complex64 = 8 B."""
    C, P, H, W = len(cfg.wavelengths), cfg.num_planes, cfg.H, cfg.W
    pH, pW = cfg.resolved_pad()
    NW = 2 * pW
    return {
        "blasm_rows": 8 * C * H * W + 8 * C * NW * pH,
        "blasm_columns": 8 * C * NW * pH + 8 * P * C * H * NW,
        "blasm_inverse_rows": 8 * P * C * H * NW + 12 * P * C * H * W,
        "loss": (4 + 4 + 4) * P * C * H * W + H * W,
        "adjoint_rows": 12 * P * C * H * W + 8 * P * C * NW * H,
        "adjoint_columns": 8 * P * C * NW * H + 8 * C * H * NW,
        "adjoint_inverse_rows": 8 * C * H * NW + 16 * C * H * W,
        "clip_adan": 44 * (7 + 2 * C) * cfg.num_gaussians,
    }


# ----------------------------------------------------------------------------------------------
# CPU reference (the oracle's torch port of the reference loop), sampled
# ----------------------------------------------------------------------------------------------
def make_cpu_pipeline(wl, seed, threads):
    from complex_valued_quadratic_phase_gaussian_b200.fit import synthetic_init
    from oracle.torch_port import ReferencePipeline
    torch.set_num_threads(threads)
    cfg = fit_config(wl, seed)
    _, _, targets, q = build_scene(wl, seed, "cpu")
    init = synthetic_init(cfg, seed)
    return ReferencePipeline({k: v.numpy() for k, v in init.items()}, (cfg.W, cfg.H), cfg.wavelengths,
                             cfg.pixel_pitch, cfg.resolved_pad(), cfg.distances(), cfg.resolved_aperture(),
                             targets.numpy(), q.numpy(), renderer="torch", device="cpu"), cfg


def cpu_sample_step(pipe, component, tiles=None):
    """Seconds one full iteration spends in `component`, measured on a bounded sample and scaled:
    render = splat fwd+bwd of a block of 64-px tiles (x total tiles / sampled tiles);
    propagate = BLASM fwd+bwd of one (plane, channel) at full size (x P*C);
    loss = multi-plane loss + SSIM fwd+bwd of one plane (x P); adan = one full Adan step."""
    if component == "render":
        rows = 1
        t0 = time.perf_counter()
        for p in pipe.params.values():
            p.grad = None
            p.requires_grad_(True)
        h = pipe.render(tile_rows=(0, rows))
        (h.real.sum() + h.imag.sum()).backward()
        return (time.perf_counter() - t0) * ((pipe.H + 63) // 64) / rows
    if component == "propagate":
        U = torch.polar(torch.rand(pipe.C, pipe.pad[0], pipe.pad[1]), torch.rand(pipe.C, pipe.pad[0], pipe.pad[1]))
        U.requires_grad_(True)
        t0 = time.perf_counter()
        pipe.propagate(U, planes=[0], channels=[0]).sum().backward()
        return (time.perf_counter() - t0) * len(pipe.dist) * pipe.C
    if component == "loss":
        I = torch.rand(1, pipe.C, pipe.H, pipe.W, requires_grad=True)
        t0 = time.perf_counter()
        pipe.loss(I, planes=[0]).backward()
        return (time.perf_counter() - t0) * len(pipe.dist)
    for p in pipe.params.values():
        if p.grad is None:
            p.grad = torch.zeros_like(p)
    t0 = time.perf_counter()
    pipe.adan_step(set(pipe.params))
    return time.perf_counter() - t0


CPU_COMPONENTS = ("render", "propagate", "loss", "adan")


def run_cpu_reference(wl, seed, rounds, warmup_rounds=1):
    """The reference CPU implementation (the oracle's torch port of the reference loop, pinned to
    the reference loop's goldens by tests/test_oracle_fit.py) on all host threads. One round = one
    bounded sample of each component (cpu_sample_step); the iteration time is the sum of the
    per-component medians over `rounds` rounds after `warmup_rounds` untimed ones, extrapolated to
    the full image / all (plane, channel) pairs / all planes."""
    threads = os.cpu_count() or 1
    pipe, cfg = make_cpu_pipeline(wl, seed, threads)
    for _ in range(warmup_rounds):
        for c in CPU_COMPONENTS:
            cpu_sample_step(pipe, c)
    samples = {c: [] for c in CPU_COMPONENTS}
    walls = []
    for _ in range(max(1, rounds)):
        t0 = time.perf_counter()
        for c in CPU_COMPONENTS:
            samples[c].append(cpu_sample_step(pipe, c))
        walls.append(time.perf_counter() - t0)
    med = {c: statistics.median(v) for c, v in samples.items()}
    spread = {c: [round(min(v), 4), round(max(v), 4)] for c, v in samples.items()}
    per_iter = sum(med.values())
    pc = len(cfg.distances()) * len(cfg.wavelengths)
    sample_desc = (f"extrapolated: per component the median of {len(walls)} bounded samples (after {warmup_rounds} "
                   f"untimed round): splat fwd+bwd on one row of 64-px tiles (x{(cfg.H + 63) // 64}), BLASM fwd+bwd "
                   f"of 1 of {pc} (plane, channel) pairs (x{pc}), loss+SSIM of 1 of {cfg.num_planes} planes "
                   f"(x{cfg.num_planes}), full Adan step; torch {torch.__version__} CPU, {threads} threads")
    return dict(value=1.0 / per_iter, cores=threads, sample=desc_trim(sample_desc), component_seconds=med,
                component_spread=spread, seconds_per_iteration=per_iter, wall_per_round=statistics.mean(walls),
                rounds=len(walls))


def desc_trim(s):
    return " ".join(s.split())


# ----------------------------------------------------------------------------------------------
# arms
# ----------------------------------------------------------------------------------------------
def run_ours(args, wl, dist, world, rank, local):
    from complex_valued_quadratic_phase_gaussian_b200.fit import Fitter, synthetic_init
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    seed = args.seed + rank
    _, _, targets, q = build_scene(wl, seed, dev, ours=True)
    cfg = fit_config(wl, seed, args.primitive)
    init = synthetic_init(cfg, seed)
    fitter = Fitter(cfg, targets, q, init=init, device=dev)
    graph = fitter.capture()
    for _ in range(args.warmup):
        graph.replay()
    # state after the warm-up: the end-to-end run below restarts from it, so that both
    # measurements cover the same iterations of the fit (the per-iteration cost grows as it fits)
    torch.cuda.synchronize()
    snap = {k: getattr(fitter, k).detach().clone() for k in ("adan_state", "iteration", "status")}
    pinned_p = fitter.flat.detach().cpu().pin_memory()
    barrier(dist)
    clocks = ClockSampler(device_smi_index(local))
    clocks.start()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(dist)
    start.record()
    for _ in range(args.steps):
        graph.replay()
    end.record()
    torch.cuda.synchronize()
    barrier(dist)
    clk = clocks.stop()
    elapsed = start.elapsed_time(end) / 1e3
    elapsed_max = max_over_ranks(dist, elapsed)
    kernels_per_step = count_graph_kernels(graph)
    launch_source = "graph kernel nodes"
    if kernels_per_step is None:
        kernels_per_step, launch_source = kernels_per_fit_step(cfg), "launch sequence of cvqpg_fit_step"
    overflow = fitter.overflowed()

    # live per-stage timing (eager launches, CUDA events on the launch stream)
    stage_ms = {}
    for _ in range(3):
        for k, v in fitter.step_timed().items():
            stage_ms.setdefault(k, []).append(v)
    stage_ms = {k: statistics.mean(v) for k, v in stage_ms.items()}
    nbytes = stage_bytes(cfg)
    hbm_stages = {k: v for k, v in stage_ms.items() if k in nbytes}
    dom = max(hbm_stages, key=hbm_stages.get)
    peak, peak_kind = measured_peaks()
    achieved = nbytes[dom] / (stage_ms[dom] / 1e3) / 1e9
    traffic = profiled_traffic(dom, args.workload)

    # end to end through the public API with pinned host buffers
    pinned_t = targets.cpu().pin_memory()
    pinned_q = q.cpu().pin_memory()
    rec = torch.empty(fitter.history.shape[1], dtype=torch.float32).pin_memory()
    out_p = torch.empty_like(pinned_p).pin_memory()
    P = cfg.num_planes
    for k, v in snap.items():  # optimiser state and counter back to the post-warm-up state
        getattr(fitter, k).copy_(v)
    it0 = int(snap["iteration"].item())
    torch.cuda.synchronize()
    barrier(dist)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.current_stream(dev)
    e0.record(stream)
    fitter.targets.copy_(pinned_t, non_blocking=True)
    fitter.depth_plane.copy_(pinned_q, non_blocking=True)
    fitter.refresh_targets()  # the job's targets arrived: noise range and SSIM moments
    fitter.flat.copy_(pinned_p, non_blocking=True)
    for i in range(args.steps):
        graph.replay()
        # the step's loss record to the host, then wait: the reference's per-iteration loss.item()
        rec.copy_(fitter.history[(it0 + i) % fitter.history.shape[0]], non_blocking=True)
        stream.synchronize()
    out_p.copy_(fitter.flat, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(dist, e0.elapsed_time(e1) / 1e3)
    h2d = (pinned_t.numel() * 4 + pinned_q.numel() + pinned_p.numel() * 4) / args.steps
    d2h = rec.numel() * 4 + pinned_p.numel() * 4 / args.steps
    ev = fitter.evaluate()

    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        ref_gpu = run_reference_gpu_sample(wl, seed, dev, steps=min(args.steps, 10), warmup=2)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = run_cpu_reference(wl, seed, rounds=3, warmup_rounds=1)
        cpu = {"value": r["value"], "unit": "it/s", "cores": r["cores"], "kind": "port", "sample": r["sample"],
               "component_seconds": {k: round(v, 4) for k, v in r["component_seconds"].items()},
               "component_spread_seconds": r["component_spread"]}

    ttp = None
    if rank == 0 and world == 1 and args.workload == "rgb1080" and not args.no_time_to_psnr:
        ttp = run_time_to_psnr()
    batched = None
    if args.batched > 0:
        batched = run_batched(args.batched, args.batched_iters, dev, dist, world, rank)

    if rank != 0:
        return None
    line = {
        "metric": METRIC, "value": world * args.steps / elapsed_max, "unit": "it/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": DATA,
        "config": workload_config(args, cfg, world),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                     "algorithmic_bytes": nbytes[dom], "ms_per_launch": stage_ms[dom]},
        "stages_ms": {k: round(v, 4) for k, v in stage_ms.items()},
        "graph": True, "fft_plan_hint": fitter.plan_hint,
        "e2e": {"value": world * args.steps / e2e_s, "unit": "it/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h),
                "note": "public Fitter API over the same iterations as the timed run (restarted from the "
                        "post-warm-up state): pinned H2D of targets/depth/params at job start, per-iteration "
                        "graph replay + loss/metric D2H with a host sync, params D2H at the end"},
        "clocks": clk,
        "gpu_launches": (kernels_per_step * args.steps) if kernels_per_step is not None else None,
        "kernels_per_step": kernels_per_step, "launch_count_source": launch_source,
        "pair_overflow": overflow,
        "psnr_after": [round(float(x), 3) for x in ev["psnr"]],
        "psnr_after_iters": int(fitter.iteration_count()),
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if ref_gpu is not None:
        line["reference_gpu"] = ref_gpu
        if "value" in ref_gpu:
            line["reference_gpu"]["ours_over_reference"] = round(line["value"] / ref_gpu["value"], 2)
    if ttp is not None:
        line["time_to_psnr"] = ttp
        plain = ttp.get("plain", {})
        if plain.get("seconds"):
            # the whole 2000-iteration fit (the per-iteration cost grows as the Gaussians spread)
            line["fit_2000_it_s"] = round(plain["iters"] / plain["seconds"], 2)
    if batched is not None:
        line["batched"] = batched
    return line


def run_batched(scenes, iters, dev, dist=None, world=1, rank=0):
    """Batched-fitter workload: `scenes` RGB scenes, a third each at 512x512, 768x1024 and
    1080x1920, with N proportional to the pixels (96k at 1080p), `iters` iterations each. The queue
    runs once through the batched fitter (one graph per iteration over the resident fits, admitted
    while their pixels stay within two 1080p images, at most 16) and once one fit at a time (1 slot),
    both timed with CUDA events on the stream that replays the graphs. With N ranks the queue is split
    by cost (batch.shard, no collective: the fits are independent) and each rank serves its share;
    the reported seconds are the maximum over the ranks."""
    from complex_valued_quadratic_phase_gaussian_b200 import scenes as S
    from complex_valued_quadratic_phase_gaussian_b200.batch import BatchedFitter, FitJob, shard
    from complex_valued_quadratic_phase_gaussian_b200.fit import FitConfig, synthetic_init
    sizes = [(512, 512), (768, 1024), (1080, 1920)]
    wl = WORKLOADS["rgb1080"]

    def jobs():
        out = []
        for i in range(scenes):
            H, W = sizes[i % 3]
            img, depth = S.rgb_blobs(H, W, seed=100 + i)
            t, q = S.multiplane_targets_device(img, depth, wl["P"], device=dev)
            n = int(round(wl["N"] * H * W / (1080 * 1920)))
            cfg = FitConfig(img_size=(W, H), num_gaussians=n, wavelengths=list(wl["wl"]), pixel_pitch=wl["pitch"],
                            num_planes=wl["P"], d_val=wl["d_val"], volume_depth=wl["vd"], num_itrs=iters, seed=i)
            out.append(FitJob(cfg, t, q, iters, init=synthetic_init(cfg, i), tag=(H, W, i)))
        return shard(out, rank, world) if world > 1 else out

    res = {}
    budget = int(2.05 * 1080 * 1920)
    for name, slots in (("batched", 16), ("serial", 1)):
        js = jobs()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = BatchedFitter(js, slots=slots, device=dev, pixel_budget=budget if slots > 1 else None).run()
        e1.record()
        torch.cuda.synchronize()
        sec = max_over_ranks(dist, e0.elapsed_time(e1) / 1e3)
        pix_it = sum(sizes[i % 3][0] * sizes[i % 3][1] for i in range(scenes)) * iters  # every rank's share
        res[name] = {"seconds": round(sec, 3), "fit_iterations_per_s": round(scenes * iters / sec, 1),
                     "megapixel_iterations_per_s": round(pix_it / sec / 1e6, 1), "slots": slots,
                     "pixel_budget": budget if slots > 1 else None,
                     "fits_done_rank0": len(out), "overflowed": sum(int(r.overflowed) for r in out)}
        del out, js
        torch.cuda.empty_cache()
    res["speedup_batched_vs_serial"] = round(res["serial"]["seconds"] / res["batched"]["seconds"], 3)
    res["workload"] = (f"{scenes} RGB scenes (512x512, 768x1024, 1080x1920 in turn; N = 96k x pixels / 1080p), "
                       f"{iters} iterations each; fit set-up (targets' moments, workspaces) inside the timed region"
                       + (f"; split over {world} ranks by cost (max over ranks)" if world > 1 else ""))
    return res


def run_time_to_psnr():
    """Second half of the metric: time for the learned-init fit to reach the plain-init fit's
    2000-iteration per-plane PSNR at 1920x1080 RGB (12 Gaussians per 16x16 tile = 97,920)."""
    from complex_valued_quadratic_phase_gaussian_b200 import learned as L
    t0 = time.time()
    w, T2, info = L.train_initialiser(num_scenes=64, H=256, W=256, iters=400, steps=3000)
    torch.cuda.synchronize()
    train_s = time.time() - t0
    res = L.time_to_psnr_experiment(w, T2, H=1080, W=1920, plain_iters=2000, eval_every=50, goal_every=1)
    res["gaussians"] = L.num_gaussians(1080, 1920)
    res["training"] = {"wall_seconds": round(train_s, 2), "pairs": info["pairs"],
                       "fits": "2 rounds x 64 fits of 256x256 crops with 1080p statistics, 400 iterations, "
                               "batched fitter; round 2 starts from round 1's network",
                       "mlp": "1024-512-512-156 GELU, BF16 tcgen05 GEMMs, FP32 Adam, 3000 steps x 8192 tiles; 10 % "
                              "of the fits held out, the weights of the best validation loss kept",
                       "final_loss": info["loss_round2"]["train"][-1][1],
                       "best_validation_loss": info["loss_round2"]["best_val"]}
    res["note"] = ("times are fit-iteration device time (CUDA events, every iteration), evaluation excluded; "
                   "the learned and constant fits are checked against the goal after every iteration; 'learned' "
                   "includes the network's prediction; 'constant' is the ablation without the network (every slot "
                   "at the mean training target)")
    return res


def run_reference_cpu_arm(args, wl, rank):
    """One step = one round of bounded component samples (cpu_sample_step); ms_per_step is the wall
    time of a round, value the extrapolated full-iteration rate."""
    if rank != 0:
        return None
    from complex_valued_quadratic_phase_gaussian_b200.fit import FitConfig  # noqa: F401 (config below)
    r = run_cpu_reference(wl, args.seed, rounds=args.steps, warmup_rounds=args.warmup)
    v = r["value"]
    cfg = fit_config(wl, args.seed, args.primitive)
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "it/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * r["wall_per_round"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": DATA,
            "config": workload_config(args, cfg, 1),
            "seconds_per_iteration_extrapolated": round(r["seconds_per_iteration"], 3),
            "cpu_baseline": {"value": v, "unit": "it/s", "cores": r["cores"], "kind": "port", "sample": r["sample"],
                             "component_seconds": {k: round(x, 4) for k, x in r["component_seconds"].items()},
                             "component_spread_seconds": r["component_spread"]},
            "e2e": {"value": v, "unit": "it/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_reference_gpu_sample(wl, seed, dev, steps, warmup):
    """The reference's GPU pipeline on the same GPU, timed outside our timed region: its own CUDA
    rasterizer (oracle/_ref, built from the reference sources) under the torch cuFFT propagator,
    loss + SSIM and Adan of the reference loop (oracle/torch_port.py), CUDA events around `steps`
    iterations after `warmup`."""
    from complex_valued_quadratic_phase_gaussian_b200.fit import synthetic_init
    from oracle.torch_port import ReferencePipeline, load_reference_extension
    ext = load_reference_extension()
    if ext is None:
        return {"unavailable": "reference CUDA extension not built (oracle/build_ref.py)"}
    cfg = fit_config(wl, seed)
    _, _, targets, q = build_scene(wl, seed, dev)
    init = synthetic_init(cfg, seed)
    torch.cuda.reset_peak_memory_stats(dev)
    pipe = ReferencePipeline({k: v.numpy() for k, v in init.items()}, (cfg.W, cfg.H), cfg.wavelengths,
                             cfg.pixel_pitch, cfg.resolved_pad(), cfg.distances(), cfg.resolved_aperture(), targets,
                             q, renderer="cuda", device=dev, ext=ext)
    for _ in range(warmup):
        pipe.step()
    torch.cuda.synchronize(dev)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(steps):
        pipe.step()
    e.record()
    torch.cuda.synchronize(dev)
    sec = s.elapsed_time(e) / 1e3
    out = {"value": round(steps / sec, 3), "unit": "it/s", "steps": steps, "warmup": warmup,
           "ms_per_step": round(1e3 * sec / steps, 3), "peak_mem_gb": round(torch.cuda.max_memory_allocated(dev) / 2 ** 30, 2),
           "pipeline": "reference cuda/ rasterizer built for sm_100a + torch cuFFT propagator, loss+SSIM, Adan "
                       "(reference loop order, per-iteration loss.item() and plane-0 PSNR on the host)"}
    del pipe
    torch.cuda.empty_cache()
    return out


def run_reference_gpu_arm(args, wl, dist, world, rank, local):
    from complex_valued_quadratic_phase_gaussian_b200.fit import synthetic_init
    from oracle.torch_port import ReferencePipeline, load_reference_extension
    ext = load_reference_extension()
    if ext is None:
        return {"impl": "reference-gpu", "unavailable": "reference CUDA extension not built (oracle/build_ref.py)"}
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    seed = args.seed + rank
    cfg = fit_config(wl, seed)
    _, _, targets, q = build_scene(wl, seed, dev)
    init = synthetic_init(cfg, seed)
    pipe = ReferencePipeline({k: v.numpy() for k, v in init.items()}, (cfg.W, cfg.H), cfg.wavelengths,
                             cfg.pixel_pitch, cfg.resolved_pad(), cfg.distances(), cfg.resolved_aperture(), targets,
                             q, renderer="cuda", device=dev, ext=ext)
    for _ in range(args.warmup):
        pipe.step()
    barrier(dist)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(args.steps):
        pipe.step()
    e.record()
    torch.cuda.synchronize()
    el = max_over_ranks(dist, s.elapsed_time(e) / 1e3)
    if rank != 0:
        return None
    return {"impl": "reference-gpu", "metric": METRIC, "value": world * args.steps / el, "unit": "it/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "dtype": "f32", "data": "synthetic",
            "config": workload_config(args, cfg, world),
            "renderer": "reference cuda/ extension built for sm_100a + torch cuFFT propagator",
            "peak_mem_gb": torch.cuda.max_memory_allocated(dev) / 2 ** 30}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-gpu"])
    ap.add_argument("--workload", default="rgb1080", choices=sorted(WORKLOADS))
    ap.add_argument("--primitive", default="curv", choices=["curv", "flat"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference GPU pipeline sample reported beside our line")
    ap.add_argument("--batched", type=int, default=0,
                    help="also run the batched-fitter workload with this many scenes (48 = the c3 case)")
    ap.add_argument("--batched-iters", type=int, default=500)
    ap.add_argument("--no-time-to-psnr", action="store_true",
                    help="skip the learned-vs-plain time-to-PSNR experiment (about a minute at N=1)")
    args = ap.parse_args()
    world, rank, local = dist_env()
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        line = run_reference_cpu_arm(args, wl, rank)
    else:
        dist = init_dist(world, local)
        try:
            if args.impl == "ours":
                line = run_ours(args, wl, dist, world, rank, local)
            else:
                line = run_reference_gpu_arm(args, wl, dist, world, rank, local)
        finally:
            if dist is not None:
                dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
