"""Autotuner for the propagation's FFT plans.

cuFFT, behind the reference propagator (utils/propagator.py:248-290), picks
its own plans; here the FFT kernels are the project's, and this module picks
their schedule per grid by measurement: the radix order of the row and column
FFTs and the radix the column kernels keep in registers between the forward
and inverse transforms (``plan_hint`` of cvqpg_blasm_params / cvqpg_fit_params).
Every distinct candidate is timed on the device (forward + adjoint
propagation, CUDA events, median of several runs); the fastest one is cached
per (grid, channels, planes, GPU) in a JSON file (``CVQPG_AUTOTUNE_CACHE``,
default ~/.cache/cvqpg_b200/autotune.json) so later fits reuse it.

The splat tile (16 x 16) and the loss tile (32 x 32) are not tuned: the
former is fixed by the reference's per-tile lists, which must match bit for bit.
"""
import json
import os
import statistics

import torch

ORDERS = (0, 1, 2, 3)
REGISTER_RADICES = (3, 5, 7, 8, 11, 13, 16)
_POW2 = {True: (16, 8), False: (8,)}


def plan_radices(n, order):
    """Radix sequence of make_fft_plan (csrc/blasm.cu) for length n and order 0..3, or None."""
    m, out = n, []

    def odd(desc):
        nonlocal m
        for r in ((17, 13, 11, 7, 5, 3) if desc else (3, 5, 7, 11, 13, 17)):
            while m % r == 0:
                out.append(r)
                m //= r

    def pow2(use16):
        nonlocal m
        for r in _POW2[use16]:
            while m % r == 0:
                out.append(r)
                m //= r
        for r in (4, 2):
            if m % r == 0:
                out.append(r)
                m //= r

    if order == 1:
        odd(True), pow2(True)
    elif order == 2:
        pow2(False), odd(False)
    elif order == 3:
        odd(True), pow2(False)
    else:
        pow2(True), odd(False)
    return out if m == 1 and len(out) <= 8 else None


def hint(col_radix=0, col_order=0, row_order=0):
    return int(col_radix) | (int(col_order) << 5) | (int(row_order) << 8)


def candidates(NH, NW):
    """Distinct plan hints for an NH x NW grid (duplicated plans removed)."""
    seen, out = set(), []
    for co in ORDERS:
        cr = plan_radices(NH, co)
        if cr is None:
            continue
        regs = sorted({r for r in cr if r in REGISTER_RADICES and (NH // r + 255) // 256 <= 2}) or [0]
        for ro in ORDERS:
            rr = plan_radices(NW, ro)
            if rr is None:
                continue
            for reg in regs:
                key = (tuple(cr), tuple(rr), reg)
                if key in seen:
                    continue
                seen.add(key)
                out.append(hint(reg, co, ro))
    return out


def _cache_path():
    return os.environ.get("CVQPG_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "cvqpg_b200", "autotune.json"))


def _load_cache():
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_cache(cache):
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home only costs a re-tune next time


def cache_key(C, P, H, W, pad, device):
    name = torch.cuda.get_device_name(device).replace(" ", "_")
    return f"{name}:C{C}:P{P}:{H}x{W}:pad{pad[0]}x{pad[1]}"


def time_hint(h, C, P, H, W, pad, wavelengths, distances, pitch, aperture, reps=5, device="cuda"):
    """Median ms of one forward + adjoint propagation with plan hint h."""
    from .propagator import BlasmPlan
    plan = BlasmPlan(C, H, W, pad, wavelengths, distances, pitch, aperture_radius=aperture, device=device,
                     plan_hint=h)
    g = torch.Generator(device=device).manual_seed(0)
    f = torch.polar(torch.rand((C, H, W), device=device, generator=g),
                    torch.rand((C, H, W), device=device, generator=g) * 6.283)
    out = plan.forward(f)
    gi = torch.empty_like(f)
    times = []
    for i in range(reps + 2):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        plan.forward(f, out=out)
        plan.backward(f, out, out=gi)
        e.record()
        torch.cuda.synchronize(device)
        if i >= 2:
            times.append(s.elapsed_time(e))
    return statistics.median(times)


def tune(C, P, H, W, pad, wavelengths, distances, pitch, aperture, reps=5, device="cuda", use_cache=True):
    """Best plan hint for this propagation geometry: (hint, {hint: ms}) (timings empty when cached)."""
    device = torch.device(device)
    key = cache_key(C, P, H, W, pad, device)
    cache = _load_cache() if use_cache else {}
    if key in cache:
        return int(cache[key]["hint"]), {}
    NH, NW = 2 * pad[0], 2 * pad[1]
    table = {}
    for h in candidates(NH, NW):
        table[h] = time_hint(h, C, P, H, W, pad, wavelengths, distances, pitch, aperture, reps, device)
    best = min(table, key=table.get)
    if use_cache:
        cache = _load_cache()
        cache[key] = {"hint": best, "ms": table[best], "default_ms": table.get(0), "candidates": len(table)}
        _store_cache(cache)
    return best, table


def tune_for(cfg, device="cuda", reps=5):
    """tune() for a FitConfig."""
    return tune(len(cfg.wavelengths), cfg.num_planes, cfg.H, cfg.W, cfg.resolved_pad(), cfg.wavelengths,
                cfg.distances(), cfg.pixel_pitch, cfg.resolved_aperture(), reps=reps, device=device)
