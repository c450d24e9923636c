"""GPU: phase-only hologram export (cvqpg_poh_encode) against the DPAC oracle.

The 8-bit levels must equal the oracle's except where float32 transcendental
rounding puts a value on the other side of a level boundary: at least 99.9 %
identical, the rest one level apart (mod 256). The reconstruction of the
8-bit hologram must be finite and resemble the targets.
"""
import numpy as np
import pytest
import torch

from oracle import poh as opoh

pytestmark = pytest.mark.gpu


def test_poh_levels_match_oracle_and_reconstruct():
    from complex_valued_quadratic_phase_gaussian_b200 import learned as L
    from complex_valued_quadratic_phase_gaussian_b200.fit import Fitter
    from complex_valued_quadratic_phase_gaussian_b200.poh import export_poh
    H, W = 96, 128
    img, depth, targets, q = L.make_scene(H, W, 11)
    cfg = L.scene_config(H, W, 150, seed=11, autotune=False)
    f = Fitter(cfg, targets, q, init=L.grid_init(cfg, 11))
    f.run(150)
    out = export_poh(f)
    field = torch.empty((3, H, W), dtype=torch.complex64, device="cuda")
    f.evaluate(field_out=field)
    pH, pW = cfg.resolved_pad()
    ref = opoh.dpac_levels(field.cpu().numpy(), pH, pW)
    got = out["levels"].cpu().numpy()
    assert got.shape == ref.shape == (3, pH, pW)
    diff = (got.astype(np.int64) - ref.astype(np.int64)) % 256
    diff = np.minimum(diff, 256 - diff)
    assert np.mean(diff == 0) >= 0.999 and diff.max() <= 1
    ph = out["phase_field"].cpu().numpy()
    assert np.allclose(np.angle(ph) % (2 * np.pi), (got.astype(np.float64) * 2 * np.pi / 256) % (2 * np.pi),
                       atol=1e-5)
    assert np.all(np.isfinite(out["psnr"])) and np.all(out["psnr"] > 5.0)


def test_poh_levels_match_reference_dpac(golden):
    """cvqpg_poh_encode against the reference's own DPAC encoding (export_poh.py:110-119, 175-180)
    of a seeded field: >= 99.9 % of the levels identical, the rest one level apart."""
    import ctypes
    from complex_valued_quadratic_phase_gaussian_b200 import _lib
    from complex_valued_quadratic_phase_gaussian_b200.propagator import BlasmPlan
    g = golden("dpac")
    field = torch.from_numpy(g["field"]).cuda()
    C, H, W = field.shape
    pH, pW = (int(v) for v in g["pad"])
    plan = BlasmPlan(C, H, W, (pH, pW), [639e-9, 515e-9, 473e-9][:C], [1e-3], 3.74e-6, device="cuda")
    levels = torch.empty((C, pH, pW), dtype=torch.uint8, device="cuda")
    _lib.check(_lib.lib().cvqpg_poh_encode(ctypes.byref(plan.params), _lib.ptr(plan.tables), plan.tables.numel(),
                                           _lib.ptr(torch.view_as_real(field)), _lib.ptr(levels), None,
                                           _lib.stream_of(torch.device("cuda"))), "cvqpg_poh_encode")
    got = levels.cpu().numpy()
    diff = (got.astype(np.int64) - g["levels"].astype(np.int64)) % 256
    diff = np.minimum(diff, 256 - diff)
    assert np.mean(diff == 0) >= 0.999 and diff.max() <= 1
