"""GPU parity of the drop-in rasterizer (binning + splat, forward and adjoint) against the oracle.

Tolerances: field 1e-5 relative L2 vs the float64 oracle on identical inputs
(the kernel computes in float32); gradients 1e-4 (float32 atomics); tile lists
and ranges bit-exact.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import splat as osp

pytestmark = pytest.mark.gpu
SPLAT_KEYS = ("means", "inv_cov", "colours", "phase", "opac", "curv", "area")


def _cuda(g, keys=SPLAT_KEYS):
    return [torch.from_numpy(np.ascontiguousarray(g[k], dtype=np.float32)).cuda() for k in keys]


def _pkg():
    import complex_valued_quadratic_phase_gaussian_b200 as pkg
    return pkg


@pytest.mark.parametrize("name", ["splat_rgb", "splat_gray"])
def test_uncut_forward_and_backward_vs_reference(golden, name):
    from complex_valued_quadratic_phase_gaussian_b200 import rasterizer as R
    g = golden(name)
    W, H = int(g["W"]), int(g["H"])
    ins = [t.requires_grad_(True) for t in _cuda(g)]
    k = torch.from_numpy(g["k"]).cuda()
    out = R.qpf_render_cull(*ins, k, float(g["dxy2"]), W, H, cull=R.CULL_NONE)
    err = rel_l2(out.detach().cpu().numpy(), g["out"])
    assert err < 1e-5, err
    gw = torch.from_numpy(g["grad_field"].astype(np.complex64)).cuda()
    out.backward(gw)
    for key, t in zip(SPLAT_KEYS, ins):
        e = rel_l2(t.grad.cpu().numpy(), g["d_" + key])
        assert e < 1e-4, (key, e)


@pytest.mark.parametrize("name", ["splat_rgb", "splat_gray"])
def test_cuda16_lists_bit_exact_and_field(golden, name):
    pkg = _pkg()
    g = golden(name)
    W, H = int(g["W"]), int(g["H"])
    cov = g["cov"]
    radii = osp.radius5_int(cov[:, 0], cov[:, 1], cov[:, 2])
    pl_ref, ranges_ref = osp.bin_lists(g["means"], W, H, osp.CULL_CUDA16_5SIGMA, radii=radii)
    ins = _cuda(g)
    k = torch.from_numpy(g["k"]).cuda()
    C = g["colours"].shape[1]
    out_r, out_i, pl, ranges = pkg.ext().qpf_render_forward(*ins, torch.from_numpy(radii).cuda(), k,
                                                            float(g["dxy2"]), W, H, C)
    assert np.array_equal(pl.cpu().numpy(), pl_ref)
    assert np.array_equal(ranges.cpu().numpy(), ranges_ref)
    ref = osp.splat_forward(*[g[k_] for k_ in SPLAT_KEYS], g["k"], float(g["dxy2"]), W, H,
                            cull=osp.CULL_CUDA16_5SIGMA, point_list=pl_ref, ranges=ranges_ref)
    got = out_r.cpu().numpy() + 1j * out_i.cpu().numpy()
    assert rel_l2(got, ref) < 1e-5
    gw = g["grad_field"]
    d = pkg.ext().qpf_render_backward(torch.from_numpy(gw.real.astype(np.float32)).cuda(),
                                      torch.from_numpy(gw.imag.astype(np.float32)).cuda(), *ins, k, pl, ranges,
                                      float(g["dxy2"]), W, H, C)
    dref = osp.splat_backward(gw, *[g[k_] for k_ in SPLAT_KEYS], g["k"], float(g["dxy2"]), W, H,
                              cull=osp.CULL_CUDA16_5SIGMA, point_list=pl_ref, ranges=ranges_ref)
    for key, a, b in zip(SPLAT_KEYS, d, dref):
        assert rel_l2(a.cpu().numpy(), b) < 1e-4, key


@pytest.mark.parametrize("name", ["torch_renderer_rgb", "torch_renderer_gray"])
def test_torch64_rule_vs_reference_torch_renderer(golden, name):
    """Gate: field within 1e-4 relative L2 of the reference PyTorch renderer (same cull rule)."""
    from complex_valued_quadratic_phase_gaussian_b200 import rasterizer as R
    g = golden(name)
    W, H = int(g["W"]), int(g["H"])
    ins = [torch.from_numpy(np.ascontiguousarray(g[k], dtype=np.float32)).cuda()
           for k in ("act_means", "act_inv_cov", "colours", "act_phase", "act_opac", "act_curv", "act_area")]
    k = torch.from_numpy(g["act_k"]).cuda()
    r3 = torch.from_numpy(g["act_radius3"]).cuda()
    out = R.qpf_render_cull(*ins, k, float(g["act_dxy2"]), W, H, cull=R.CULL_TORCH64_3SIGMA, radius3=r3)
    got = out.cpu().numpy()
    assert rel_l2(got, g["field"]) < 1e-4
    pl_ref, ranges_ref = osp.bin_lists(g["act_means"], W, H, osp.CULL_TORCH64_3SIGMA, radius3=g["act_radius3"])
    ref64 = osp.splat_forward(g["act_means"], g["act_inv_cov"], g["colours"], g["act_phase"], g["act_opac"],
                              g["act_curv"], g["act_area"], g["act_k"], float(g["act_dxy2"]), W, H,
                              cull=osp.CULL_TORCH64_3SIGMA, point_list=pl_ref, ranges=ranges_ref)
    assert rel_l2(got, ref64) < 1e-5


def test_c0_scale_lists_bit_exact():
    """256x256, N=4096 (the grayscale fit size): lists and ranges bit-exact vs the oracle."""
    pkg = _pkg()
    rng = np.random.default_rng(5)
    n, W, H = 4096, 256, 256
    means = np.stack([rng.uniform(-8, W + 8, n), rng.uniform(-8, H + 8, n)], 1).astype(np.float32)
    radii = np.ceil(5 * (np.exp(rng.normal(np.log(2.0), 0.3, n)) + 0.1)).astype(np.int32)
    radii[::97] = 0
    radii[::89] = 40
    pl_ref, ranges_ref = osp.bin_lists(means, W, H, osp.CULL_CUDA16_5SIGMA, radii=radii)
    z = torch.zeros(n, device="cuda")
    inv = torch.tensor([0.2, 0.0, 0.2], device="cuda").repeat(n, 1)
    ones = torch.ones(n, 1, device="cuda")
    k = torch.tensor([2 * np.pi / 515e-9], dtype=torch.float32, device="cuda")
    _, _, pl, ranges = pkg.ext().qpf_render_forward(torch.from_numpy(means).cuda(), inv, ones, ones * 0, z + 0.5, z,
                                                    z + 4, torch.from_numpy(radii).cuda(), k, 6.4e-11, W, H, 1)
    assert np.array_equal(pl.cpu().numpy(), pl_ref)
    assert np.array_equal(ranges.cpu().numpy(), ranges_ref)


def test_capacity_retry_and_empty():
    from complex_valued_quadratic_phase_gaussian_b200 import rasterizer as R
    rng = np.random.default_rng(6)
    n, W, H = 500, 64, 48
    means = torch.from_numpy(np.stack([rng.uniform(0, W, n), rng.uniform(0, H, n)], 1).astype(np.float32)).cuda()
    inv = torch.tensor([0.2, 0.0, 0.2], device="cuda").repeat(n, 1)
    ones = torch.ones(n, 3, device="cuda")
    z = torch.zeros(n, device="cuda")
    radii = torch.full((n,), 30, dtype=torch.int32, device="cuda")
    k = torch.tensor([1e7, 1.2e7, 1.3e7], device="cuda")
    R._capacity_hint[(n, W, H, R.CULL_CUDA16_5SIGMA)] = 16  # force the overflow/retry path
    out1, pl1, _ = R.render_forward(means, inv, ones, ones, z + 0.5, z, z + 4, k, 1e-11, W, H, radii=radii)
    out2, pl2, _ = R.render_forward(means, inv, ones, ones, z + 0.5, z, z + 4, k, 1e-11, W, H, radii=radii)
    assert torch.equal(pl1, pl2) and pl1.numel() > 16
    assert torch.allclose(out1, out2)
    # zero Gaussians: zero field, one-element list (cuda/raster.cu:72-75)
    e = torch.zeros(0, 2, device="cuda")
    out, pl, ranges = R.render_forward(e, torch.zeros(0, 3, device="cuda"), torch.zeros(0, 3, device="cuda"),
                                       torch.zeros(0, 3, device="cuda"), torch.zeros(0, device="cuda"),
                                       torch.zeros(0, device="cuda"), torch.zeros(0, device="cuda"), k, 1e-11, W, H,
                                       radii=torch.zeros(0, dtype=torch.int32, device="cuda"))
    assert out.abs().max().item() == 0 and pl.numel() == 1 and ranges.abs().max().item() == 0


def test_reference_error_behaviour():
    pkg = _pkg()
    n = 4
    t = lambda *s: torch.zeros(*s, device="cuda")
    radii = torch.ones(n, dtype=torch.int32, device="cuda")
    with pytest.raises(RuntimeError, match="1 or 3 channels"):
        pkg.ext().qpf_render_forward(t(n, 2), t(n, 3), t(n, 2), t(n, 2), t(n), t(n), t(n), radii, t(2), 1.0, 8, 8, 2)
    with pytest.raises(RuntimeError, match="must be contiguous"):
        pkg.ext().qpf_render_forward(t(2, n).t(), t(n, 3), t(n, 1), t(n, 1), t(n), t(n), t(n), radii, t(1), 1.0,
                                     8, 8, 1)
    with pytest.raises(RuntimeError, match="must be CUDA"):
        pkg.ext().qpf_render_forward(torch.zeros(n, 2), t(n, 3), t(n, 1), t(n, 1), t(n), t(n), t(n), radii, t(1),
                                     1.0, 8, 8, 1)
    with pytest.raises(RuntimeError, match="rows, expected"):
        pkg.ext().qpf_render_forward(t(n, 2), t(n + 1, 3), t(n, 1), t(n, 1), t(n), t(n), t(n), radii, t(1), 1.0,
                                     8, 8, 1)
    with pytest.raises(RuntimeError, match="num_channels entries"):
        pkg.ext().qpf_render_forward(t(n, 2), t(n, 3), t(n, 1), t(n, 1), t(n), t(n), t(n), radii, t(3), 1.0, 8, 8,
                                     1)


def test_isotropic_phase_vs_reference_torch_renderer(golden):
    """--phase_iso (the reference supports it only in its torch renderer): field within 1e-4 of that
    renderer, within 1e-5 of the float64 oracle; adjoint within 1e-4 of the oracle, no area gradient."""
    from complex_valued_quadratic_phase_gaussian_b200 import rasterizer as R
    g = golden("torch_renderer_iso_rgb")
    W, H = int(g["W"]), int(g["H"])
    names = ("act_means", "act_inv_cov", "colours", "act_phase", "act_opac", "act_curv", "act_area")
    ins = [torch.from_numpy(np.ascontiguousarray(g[k], dtype=np.float32)).cuda().requires_grad_(True) for k in names]
    k = torch.from_numpy(g["act_k"]).cuda()
    r3 = torch.from_numpy(g["act_radius3"]).cuda()
    out = R.qpf_render_cull(*ins, k, float(g["act_dxy2"]), W, H, cull=R.CULL_TORCH64_3SIGMA, radius3=r3,
                            phase_iso=True)
    got = out.detach().cpu().numpy()
    assert rel_l2(got, g["field"]) < 1e-4
    args = [g[k_] for k_ in names]
    pl, ranges = osp.bin_lists(g["act_means"], W, H, osp.CULL_TORCH64_3SIGMA, radius3=g["act_radius3"])
    ref = osp.splat_forward(*args, g["act_k"], float(g["act_dxy2"]), W, H, cull=osp.CULL_TORCH64_3SIGMA,
                            point_list=pl, ranges=ranges, phase_iso=True)
    assert rel_l2(got, ref) < 1e-5
    gw = g["grad_field"]  # any fixed field-shaped weight
    gt = torch.from_numpy(gw.astype(np.complex64)).cuda()
    ((out.real * gt.real).sum() + (out.imag * gt.imag).sum()).backward()
    dref = osp.splat_backward(gw, *args, g["act_k"], float(g["act_dxy2"]), W, H, cull=osp.CULL_TORCH64_3SIGMA,
                              point_list=pl, ranges=ranges, phase_iso=True)
    for name, t, b in zip(names, ins, dref):
        if name == "act_area":
            assert torch.count_nonzero(t.grad).item() == 0
            continue
        assert rel_l2(t.grad.cpu().numpy(), b) < 1e-4, name


@pytest.mark.parametrize("iso", [False, True])
def test_adjoint_thin_gaussians_ragged_tiles_vs_float64_oracle(iso):
    """The splat adjoint works on per-row spans of the Mahalanobis cut (length-sorted segments).
    Thin, rotated Gaussians (spans of a pixel or two, rows with none), Gaussians past the image
    border and a 70 x 45 image (ragged edge tiles) against the float64 oracle on the same lists:
    every gradient within 1e-4 relative L2."""
    from complex_valued_quadratic_phase_gaussian_b200.rasterizer import render_backward, render_forward
    rng = np.random.default_rng(21 + iso)
    n, W, H, C = 300, 70, 45, 3
    means = np.stack([rng.uniform(-8, W + 8, n), rng.uniform(-8, H + 8, n)], 1).astype(np.float32)
    s = np.stack([rng.uniform(0.35, 0.8, n), rng.uniform(3.0, 9.0, n)], 1)  # aspect up to ~25
    th = rng.uniform(0, np.pi, n)
    c, si = np.cos(th), np.sin(th)
    c00 = s[:, 0] ** 2 * c * c + s[:, 1] ** 2 * si * si + 0.1
    c01 = (s[:, 0] ** 2 - s[:, 1] ** 2) * c * si
    c11 = s[:, 0] ** 2 * si * si + s[:, 1] ** 2 * c * c + 0.1
    det = c00 * c11 - c01 ** 2
    inv = np.stack([c11 / det, -c01 / det, c00 / det], 1).astype(np.float32)
    radii = osp.radius5_int(c00, c01, c11)
    col = rng.uniform(0, 1, (n, C)).astype(np.float32)
    ph = rng.uniform(0, 2 * np.pi, (n, C)).astype(np.float32)
    op = rng.uniform(0.2, 0.9, n).astype(np.float32)
    cv = rng.normal(0, 800, n).astype(np.float32)
    ar = (s[:, 0] * s[:, 1]).astype(np.float32)
    k = (2 * np.pi / np.array([639e-9, 515e-9, 473e-9])).astype(np.float32)
    dxy2 = 3.74e-6 ** 2
    T = [torch.from_numpy(a).cuda() for a in (means, inv, col, ph, op, cv, ar)]
    K = torch.from_numpy(k).cuda()
    R = torch.from_numpy(radii).cuda()
    _, pl, ranges = render_forward(*T, K, dxy2, W, H, radii=R, phase_iso=iso)
    g = (rng.normal(size=(C, H, W)) + 1j * rng.normal(size=(C, H, W))).astype(np.complex64)
    got = render_backward(torch.from_numpy(g).cuda(), *T, K, pl, ranges, dxy2, W, H, phase_iso=iso)
    ref = osp.splat_backward(g, means, inv, col, ph, op, cv, ar, k, dxy2, W, H, cull=osp.CULL_CUDA16_5SIGMA,
                             point_list=pl.cpu().numpy(), ranges=ranges.cpu().numpy().reshape(-1, 2),
                             phase_iso=iso)
    names = ("d_means", "d_inv", "d_col", "d_ph", "d_op", "d_cv", "d_ar")
    for name, a, b in zip(names, got, ref):
        a = a.cpu().numpy().astype(np.float64).reshape(b.shape)
        if iso and name == "d_ar":
            continue  # the isotropic phase does not use the area
        assert rel_l2(a, b) < 1e-4, (name, rel_l2(a, b))


@pytest.mark.parametrize("C,iso", [(3, False), (1, False), (3, True)])
def test_adjoint_long_lists_over_many_batches_vs_float64_oracle(C, iso):
    """Tiles whose lists hold several batches of entries (the adjoint stages 96 per batch): 700
    Gaussians of 0.6-5 px, 500 of them within 10 px of one point, so the tiles around it list
    hundreds of entries, the same Gaussian often several times per batch in one warp's segments.
    Large curvatures (the phase turns quickly along a row). Every gradient within 1e-4 relative L2
    of the float64 oracle on the same lists, and the lists are those of the oracle's binning."""
    from complex_valued_quadratic_phase_gaussian_b200.rasterizer import render_backward, render_forward
    rng = np.random.default_rng(7 + C + 10 * iso)
    n, W, H = 700, 80, 56
    centre = np.array([37.0, 29.0])
    means = np.concatenate([centre + rng.normal(0, 5.0, (500, 2)),
                            np.stack([rng.uniform(0, W, 200), rng.uniform(0, H, 200)], 1)]).astype(np.float32)
    s = rng.uniform(0.6, 5.0, (n, 2))
    th = rng.uniform(0, np.pi, n)
    c, si = np.cos(th), np.sin(th)
    c00 = s[:, 0] ** 2 * c * c + s[:, 1] ** 2 * si * si + 0.05
    c01 = (s[:, 0] ** 2 - s[:, 1] ** 2) * c * si
    c11 = s[:, 0] ** 2 * si * si + s[:, 1] ** 2 * c * c + 0.05
    det = c00 * c11 - c01 ** 2
    inv = np.stack([c11 / det, -c01 / det, c00 / det], 1).astype(np.float32)
    radii = osp.radius5_int(c00, c01, c11)
    col = rng.uniform(0, 1, (n, C)).astype(np.float32)
    ph = rng.uniform(0, 2 * np.pi, (n, C)).astype(np.float32)
    op = rng.uniform(0.2, 0.9, n).astype(np.float32)
    cv = rng.normal(0, 1500, n).astype(np.float32)
    ar = (s[:, 0] * s[:, 1]).astype(np.float32)
    wl = [639e-9, 515e-9, 473e-9][:C] if C == 3 else [515e-9]
    k = (2 * np.pi / np.array(wl)).astype(np.float32)
    dxy2 = 3.74e-6 ** 2
    T = [torch.from_numpy(a).cuda() for a in (means, inv, col, ph, op, cv, ar)]
    K = torch.from_numpy(k).cuda()
    _, pl, ranges = render_forward(*T, K, dxy2, W, H, radii=torch.from_numpy(radii).cuda(), phase_iso=iso)
    pl_ref, ranges_ref = osp.bin_lists(means, W, H, osp.CULL_CUDA16_5SIGMA, radii=radii)
    assert np.array_equal(pl.cpu().numpy()[:len(pl_ref)], pl_ref)
    lens = ranges_ref[:, 1] - ranges_ref[:, 0]
    assert lens.max() > 3 * 96, lens.max()
    g = (rng.normal(size=(C, H, W)) + 1j * rng.normal(size=(C, H, W))).astype(np.complex64)
    got = render_backward(torch.from_numpy(g).cuda(), *T, K, pl, ranges, dxy2, W, H, phase_iso=iso)
    ref = osp.splat_backward(g, means, inv, col, ph, op, cv, ar, k, dxy2, W, H, cull=osp.CULL_CUDA16_5SIGMA,
                             point_list=pl_ref, ranges=ranges_ref, phase_iso=iso)
    names = ("d_means", "d_inv", "d_col", "d_ph", "d_op", "d_cv", "d_ar")
    for name, a, b in zip(names, got, ref):
        if iso and name == "d_ar":
            continue
        a = a.cpu().numpy().astype(np.float64).reshape(b.shape)
        e = rel_l2(a, b)
        print(f"long lists C={C} iso={iso} {name}: rel-L2 {e:.2e}")
        assert e < 1e-4, (name, e)
