"""GPU parity of the fused pad/clamp/BLASM kernels and their adjoint.

Gates: per-plane intensity within 1e-4 relative L2 of the reference propagator
chain (golden fixtures); complex field within 2e-5 of the float64 oracle;
gradients within 1e-4 of the reference autograd.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import blasm as ob

pytestmark = pytest.mark.gpu
CASES = ["propagate_rgb", "propagate_gray_bandlimit"]


def _plan(g, **kw):
    from complex_valued_quadratic_phase_gaussian_b200.propagator import BlasmPlan
    C, H, W = g["field"].shape
    return BlasmPlan(C, H, W, (int(g["pH"]), int(g["pW"])), list(g["wavelengths"]), list(g["distances"]),
                     float(g["pitch"]), aperture_radius=float(g["aperture"]), **kw)


def _oargs(g):
    return int(g["pH"]), int(g["pW"]), list(g["wavelengths"]), list(g["distances"]), float(g["pitch"])


@pytest.mark.parametrize("name", CASES)
def test_forward_and_adjoint_vs_reference(golden, name):
    g = golden(name)
    plan = _plan(g)
    field = torch.from_numpy(g["field"]).cuda()
    V = plan.forward(field)
    Vn = V.cpu().numpy()
    assert rel_l2(np.abs(Vn) ** 2, g["I_crop"]) < 1e-4
    pH, pW, wl, dist, dx = _oargs(g)
    Vo = ob.chain_forward(g["field"].astype(np.complex128), pH, pW, wl, dist, dx, aperture_radius=float(g["aperture"]))
    assert rel_l2(Vn, Vo) < 2e-5
    gV = (2.0 * V * torch.from_numpy(g["wts"]).cuda()).contiguous()
    gf = plan.backward(field, gV).cpu().numpy()
    assert rel_l2(gf, g["grad_field"]) < 1e-4
    go = ob.chain_backward(g["field"].astype(np.complex128), 2.0 * Vo * g["wts"], pH, pW, wl, dist, dx,
                           aperture_radius=float(g["aperture"]))
    assert rel_l2(gf, go) < 2e-5
    assert gf[0, 3, 5] == 0


@pytest.mark.parametrize("name", CASES)
def test_reference_propagator_class_full_output(golden, name):
    from complex_valued_quadratic_phase_gaussian_b200.propagator import propagator
    g = golden(name)
    pH, pW, wl, dist, dx = _oargs(g)
    C = g["field"].shape[0]
    U = ob.soft_window_pad(g["field"].astype(np.complex128), pH, pW)
    phase = torch.from_numpy(np.mod(np.angle(U), 2 * np.pi).astype(np.float32)).cuda()
    amp = torch.from_numpy(np.clip(np.abs(U), 0, 1).astype(np.float32)).cuda()
    prop = propagator(resolution=[pH, pW], wavelengths=wl, pixel_pitch=dx, number_of_frames=C,
                      distances=torch.tensor(dist, dtype=torch.float64), laser_channel_power=torch.eye(C),
                      aperture_size=float(g["aperture"]), device=torch.device("cuda"))
    I = prop.reconstruct(phase, amplitude=amp).sum(0).cpu().numpy()
    assert rel_l2(I, g["I_full"]) < 1e-4


def _random_field(rng, C, H, W):
    a = rng.uniform(0, 1.3, (C, H, W))
    return (a * np.exp(1j * rng.uniform(0, 2 * np.pi, (C, H, W)))).astype(np.complex64)


def test_grayscale_256_three_planes_vs_oracle_and_adjoint():
    """The 256x256 grayscale geometry (pad 576, FFT 1152 = 2^7 * 9, planes 1.0/1.5/2.0 mm)."""
    from complex_valued_quadratic_phase_gaussian_b200.propagator import BlasmPlan, reference_distances
    rng = np.random.default_rng(1)
    H = W = 256
    dist = reference_distances(3, 1e-3, 1.5e-3)
    plan = BlasmPlan(1, H, W, (576, 576), [515e-9], dist, 8e-6, aperture_radius=2560)
    f = _random_field(rng, 1, H, W)
    V = plan.forward(torch.from_numpy(f).cuda())
    Vo = ob.chain_forward(f.astype(np.complex128), 576, 576, [515e-9], dist, 8e-6, aperture_radius=2560)
    assert rel_l2(V.cpu().numpy(), Vo) < 2e-5
    y = (rng.normal(size=V.shape) + 1j * rng.normal(size=V.shape)).astype(np.complex64)
    # adjoint identity of the linear part (input mode 1 = no clamp)
    plan1 = BlasmPlan(1, H, W, (576, 576), [515e-9], dist, 8e-6, aperture_radius=2560, input_mode=1)
    x = _random_field(rng, 1, 576, 576)
    Lx = plan1.forward(torch.from_numpy(x).cuda()).cpu().numpy().astype(np.complex128)
    Lty = plan1.backward(None, torch.from_numpy(y).cuda()).cpu().numpy().astype(np.complex128)
    lhs, rhs = np.vdot(y.astype(np.complex128), Lx), np.vdot(Lty, x.astype(np.complex128))
    assert abs(lhs - rhs) < 1e-4 * abs(lhs)


def test_rgb_1080p_three_planes_vs_oracle():
    """1920x1080 RGB headline geometry: pad 1408x2240, FFT grid 2816 x 4480, 3 planes."""
    from complex_valued_quadratic_phase_gaussian_b200.propagator import (BlasmPlan, reference_distances,
                                                                         reference_pad_size)
    rng = np.random.default_rng(2)
    H, W = 1080, 1920
    pad = reference_pad_size((W, H))
    assert pad == [1408, 2240]
    wl = [639e-9, 515e-9, 473e-9]
    dist = reference_distances(3, 1e-3, 1e-3)
    plan = BlasmPlan(3, H, W, pad, wl, dist, 3.74e-6, aperture_radius=19200)
    f = _random_field(rng, 3, H, W)
    V = plan.forward(torch.from_numpy(f).cuda()).cpu().numpy()
    Vo = ob.chain_forward(f.astype(np.complex128), pad[0], pad[1], wl, dist, 3.74e-6, aperture_radius=19200)
    assert rel_l2(V, Vo) < 2e-5
    gV = (rng.normal(size=V.shape) + 1j * rng.normal(size=V.shape)).astype(np.complex64)
    gf = plan.backward(torch.from_numpy(f).cuda(), torch.from_numpy(gV).cuda()).cpu().numpy()
    go = ob.chain_backward(f.astype(np.complex128), gV.astype(np.complex128), pad[0], pad[1], wl, dist, 3.74e-6,
                           aperture_radius=19200)
    assert rel_l2(gf, go) < 2e-5


def test_rgb_1080p_compile_time_plans_match_run_time_plans():
    """At the 1080p grid (2816 x 4480) the default plan runs the kernels whose FFT passes are fixed
    at compile time (columns: four adjacent columns per CTA, 16 x 11 x 16 with the last radix 16
    in registers; rows 16 x 8 x 5 x 7). plan_hint CVQPG_PLAN_COLS1 runs the one-column compile-time
    kernels (16 x 16 x 11, radix 11 in registers), plan_hint 16 (radix 16 in registers, one
    column) the run-time column plan, plan_hint 2 << 8 (row radices 8/4/2 first) the run-time row
    plan. Forward and adjoint agree within 1e-5 relative L2."""
    from complex_valued_quadratic_phase_gaussian_b200.propagator import (BlasmPlan, reference_distances,
                                                                         reference_pad_size)
    rng = np.random.default_rng(5)
    H, W = 1080, 1920
    pad = reference_pad_size((W, H))
    wl = [639e-9, 515e-9, 473e-9]
    dist = reference_distances(3, 1e-3, 1e-3)
    a = BlasmPlan(3, H, W, pad, wl, dist, 3.74e-6, aperture_radius=19200)
    b = BlasmPlan(3, H, W, pad, wl, dist, 3.74e-6, aperture_radius=19200, plan_hint=16)
    f = torch.from_numpy(_random_field(rng, 3, H, W)).cuda()
    g = torch.from_numpy((rng.normal(size=(3, 3, H, W)) + 1j * rng.normal(size=(3, 3, H, W))).astype(np.complex64))
    g = g.cuda()
    c = BlasmPlan(3, H, W, pad, wl, dist, 3.74e-6, aperture_radius=19200, plan_hint=2 << 8)
    d = BlasmPlan(3, H, W, pad, wl, dist, 3.74e-6, aperture_radius=19200, plan_hint=1 << 11)
    va, vb, vc, vd = (p.forward(f).cpu().numpy() for p in (a, b, c, d))
    ga, gb, gc, gd = (p.backward(f, g).cpu().numpy() for p in (a, b, c, d))
    assert rel_l2(va, vb) < 1e-5 and rel_l2(va, vc) < 1e-5 and rel_l2(va, vd) < 1e-5
    assert rel_l2(ga, gb) < 1e-5 and rel_l2(ga, gc) < 1e-5 and rel_l2(ga, gd) < 1e-5


def test_rgb_1080p_padded_input_four_and_one_column_kernels_agree():
    """input_mode 1 (an already padded field, as the POH reconstruction uses) with the full padded
    output at the 1080p grid: the four-column kernels keep every row of the middle half; forward and
    adjoint agree with the one-column kernels (CVQPG_PLAN_COLS1) within 1e-5 relative L2. With 1408
    kept rows the four-column adjoint reads each plane's input straight from global memory (the
    fit's 1080-row crops are staged in shared memory instead, covered by the fit and BLASM tests)."""
    from complex_valued_quadratic_phase_gaussian_b200.propagator import (BlasmPlan, reference_distances,
                                                                         reference_pad_size)
    rng = np.random.default_rng(8)
    H, W = 1080, 1920
    pH, pW = reference_pad_size((W, H))
    wl = [639e-9, 515e-9, 473e-9]
    dist = reference_distances(3, 1e-3, 1e-3)
    kw = dict(aperture_radius=min(W, H), out_size=(pH, pW), input_mode=1)
    a = BlasmPlan(3, H, W, (pH, pW), wl, dist, 3.74e-6, **kw)
    b = BlasmPlan(3, H, W, (pH, pW), wl, dist, 3.74e-6, plan_hint=1 << 11, **kw)
    f = torch.from_numpy(_random_field(rng, 3, pH, pW)).cuda()
    g = torch.from_numpy((rng.normal(size=(3, 3, pH, pW)) + 1j * rng.normal(size=(3, 3, pH, pW))).astype(np.complex64))
    g = g.cuda()
    assert rel_l2(a.forward(f).cpu().numpy(), b.forward(f).cpu().numpy()) < 1e-5
    assert rel_l2(a.backward(f, g).cpu().numpy(), b.backward(f, g).cpu().numpy()) < 1e-5


@pytest.mark.parametrize("H,W,col_hint", [(512, 512, 16), (768, 1024, 8), (256, 256, 16)])
def test_compile_time_plans_of_the_other_grids_match_run_time_plans(H, W, col_hint):
    """The compile-time FFT plans of the 512x512 (1664^2), 768x1024 (2176 x 2688) and 256x256
    (1152^2) grids against the run-time plans of the same grids: `col_hint` moves the column split
    off the compiled one, plan_hint 2 << 8 the row radix order. Within 1e-5 relative L2."""
    from complex_valued_quadratic_phase_gaussian_b200.propagator import (BlasmPlan, reference_distances,
                                                                         reference_pad_size)
    rng = np.random.default_rng(H + W)
    pad = reference_pad_size((W, H))
    wl = [639e-9, 515e-9, 473e-9]
    dist = reference_distances(3, 1e-3, 1e-3)
    plans = [BlasmPlan(3, H, W, pad, wl, dist, 3.74e-6, aperture_radius=10 * max(H, W), plan_hint=h)
             for h in (0, col_hint, 2 << 8)]
    f = torch.from_numpy(_random_field(rng, 3, H, W)).cuda()
    g = torch.from_numpy((rng.normal(size=(3, 3, H, W)) + 1j * rng.normal(size=(3, 3, H, W))).astype(np.complex64))
    g = g.cuda()
    v = [p.forward(f).cpu().numpy() for p in plans]
    a = [p.backward(f, g).cpu().numpy() for p in plans]
    for i in (1, 2):
        assert rel_l2(v[0], v[i]) < 1e-5, (i, rel_l2(v[0], v[i]))
        assert rel_l2(a[0], a[i]) < 1e-5, (i, rel_l2(a[0], a[i]))
