"""GPU: every FFT plan the autotuner may pick gives the same propagation.

Each candidate plan hint (radix order of the row and column FFTs, radix held in
registers by the column kernels) must reproduce the default plan's forward
intensity field and adjoint within 1e-5 relative L2 (float32 FFTs with
different rounding order); tune() must return one of them and cache it.
"""
import json

import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def test_all_candidate_plans_agree(tmp_path, monkeypatch):
    from complex_valued_quadratic_phase_gaussian_b200 import autotune
    from complex_valued_quadratic_phase_gaussian_b200.propagator import BlasmPlan
    C, H, W, pad = 3, 96, 128, (176, 240)            # FFT grid 352 x 480 = (2^5 11) x (2^5 3 5)
    wl, dist, pitch = [639e-9, 515e-9, 473e-9], [0.5e-3, 1e-3, 1.5e-3], 3.74e-6
    g = torch.Generator(device="cuda").manual_seed(3)
    f = torch.polar(torch.rand((C, H, W), device="cuda", generator=g) * 1.2,
                    torch.rand((C, H, W), device="cuda", generator=g) * 6.283)
    go = torch.polar(torch.rand((3, C, H, W), device="cuda", generator=g),
                     torch.rand((3, C, H, W), device="cuda", generator=g) * 6.283)
    ref = BlasmPlan(C, H, W, pad, wl, dist, pitch, aperture_radius=200)
    v0, a0 = ref.forward(f), ref.backward(f, go)
    hints = autotune.candidates(2 * pad[0], 2 * pad[1])
    assert len(hints) > 8
    for h in hints:
        p = BlasmPlan(C, H, W, pad, wl, dist, pitch, aperture_radius=200, plan_hint=h)
        v, a = p.forward(f), p.backward(f, go)
        torch.cuda.synchronize()
        assert rel_l2(v.cpu().numpy(), v0.cpu().numpy()) < 1e-5, h
        assert rel_l2(a.cpu().numpy(), a0.cpu().numpy()) < 1e-5, h
    cache = tmp_path / "tune.json"
    monkeypatch.setenv("CVQPG_AUTOTUNE_CACHE", str(cache))
    best, table = autotune.tune(C, 3, H, W, pad, wl, dist, pitch, 200, reps=2)
    assert best in hints and set(table) == set(hints)
    assert json.loads(cache.read_text())[autotune.cache_key(C, 3, H, W, pad, torch.device("cuda"))]["hint"] == best
    assert autotune.tune(C, 3, H, W, pad, wl, dist, pitch, 200) == (best, {})
