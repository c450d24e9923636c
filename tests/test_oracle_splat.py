"""CPU: pin the splat / binning / preprocessing oracle against the reference's own outputs."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import preprocess as opre
from oracle import splat as osp

SPLAT_KEYS = ("means", "inv_cov", "colours", "phase", "opac", "curv", "area")


@pytest.mark.parametrize("name", ["splat_rgb", "splat_gray"])
def test_oracle_uncut_forward_matches_reference(golden, name):
    g = golden(name)
    out = osp.splat_forward(*[g[k] for k in SPLAT_KEYS], g["k"], float(g["dxy2"]), int(g["W"]), int(g["H"]),
                            cull=osp.CULL_NONE)
    assert rel_l2(out, g["out"]) < 1e-12


@pytest.mark.parametrize("name", ["splat_rgb", "splat_gray"])
def test_oracle_uncut_backward_matches_reference_autograd(golden, name):
    g = golden(name)
    grads = osp.splat_backward(g["grad_field"], *[g[k] for k in SPLAT_KEYS], g["k"], float(g["dxy2"]),
                               int(g["W"]), int(g["H"]), cull=osp.CULL_NONE)
    for key, got in zip(SPLAT_KEYS, grads):
        assert rel_l2(got, g["d_" + key]) < 1e-10, key


def test_cuda16_lists_are_sorted_rect_covers(golden):
    g = golden("splat_rgb")
    W, H = int(g["W"]), int(g["H"])
    cov = g["cov"]
    radii = osp.radius5_int(cov[:, 0], cov[:, 1], cov[:, 2])
    pl, ranges = osp.bin_lists(g["means"], W, H, osp.CULL_CUDA16_5SIGMA, radii=radii)
    gx, gy = (W + 15) // 16, (H + 15) // 16
    total = 0
    for t in range(gx * gy):
        s, e = ranges[t]
        ids = pl[s:e]
        assert np.all(np.diff(ids) > 0)
        for i in ids:
            x0, y0, x1, y1 = osp.tile_rect_f32(g["means"][i, 0], g["means"][i, 1], radii[i], gx, gy)
            assert x0 <= t % gx < x1 and y0 <= t // gx < y1
        total += e - s
    expect = 0
    for i in range(g["means"].shape[0]):
        x0, y0, x1, y1 = osp.tile_rect_f32(g["means"][i, 0], g["means"][i, 1], radii[i], gx, gy)
        expect += max(0, x1 - x0) * max(0, y1 - y0)
    assert total == expect


def test_cuda16_cull_close_to_uncut(golden):
    g = golden("splat_rgb")
    W, H = int(g["W"]), int(g["H"])
    cov = g["cov"]
    radii = osp.radius5_int(cov[:, 0], cov[:, 1], cov[:, 2])
    pl, ranges = osp.bin_lists(g["means"], W, H, osp.CULL_CUDA16_5SIGMA, radii=radii)
    out = osp.splat_forward(*[g[k] for k in SPLAT_KEYS], g["k"], float(g["dxy2"]), W, H,
                            cull=osp.CULL_CUDA16_5SIGMA, point_list=pl, ranges=ranges)
    assert rel_l2(out, g["out"]) < 2e-4  # 5-sigma rectangle drops < exp(-12.5) per Gaussian


@pytest.mark.parametrize("name", ["torch_renderer_rgb", "torch_renderer_gray"])
def test_oracle_torch64_matches_reference_torch_renderer(golden, name):
    g = golden(name)
    W, H = int(g["W"]), int(g["H"])
    pl, ranges = osp.bin_lists(g["act_means"], W, H, osp.CULL_TORCH64_3SIGMA, radius3=g["act_radius3"])
    out = osp.splat_forward(g["act_means"], g["act_inv_cov"], g["colours"], g["act_phase"], g["act_opac"],
                            g["act_curv"], g["act_area"], g["act_k"], float(g["act_dxy2"]), W, H,
                            cull=osp.CULL_TORCH64_3SIGMA, point_list=pl, ranges=ranges)
    # the reference computes in float32; the oracle in float64
    assert rel_l2(out, g["field"]) < 2e-6


@pytest.mark.parametrize("name", ["preprocess_rgb", "preprocess_gray"])
@pytest.mark.parametrize("mode", ["scale_aware", "constant", "off"])
def test_oracle_preprocess_matches_reference(golden, name, mode):
    g = golden(name)
    W, H, C = int(g["W"]), int(g["H"]), int(g["C"])
    raw = {k: g[k] for k in opre.RAW_KEYS}
    wl = [639e-9, 515e-9, 473e-9][:C] if C == 3 else [639e-9]
    act = opre.activate(raw, W, H, wl, 3.74e-6, curv_mode=mode)
    for key in ("means", "inv_cov", "phase", "opac", "curv", "area", "cov"):
        ref = g[f"{mode}__{key}"]
        tol = 1e-5 if key != "phase" else 1e-6
        if key == "curv" and mode == "off":
            assert np.all(act[key] == 0) and np.all(ref == 0)
            continue
        assert rel_l2(act[key], ref) < tol, key
    cov = g[f"{mode}__cov"]
    assert np.array_equal(osp.radius5_int(cov[:, 0], cov[:, 1], cov[:, 2]), g[f"{mode}__radii"])
    # torch's CPU float32 sqrt is 0.5001-ulp (near-ties can round the other way); allow 2 ulp after the x3
    r3 = osp.radius3_float(cov[:, 0], cov[:, 1], cov[:, 2])
    assert np.all(np.abs(r3 - g[f"{mode}__radius3"]) <= 2 * np.spacing(g[f"{mode}__radius3"]))
    # chain rule against torch autograd of the reference
    w = {k: g[f"{mode}__w_{k}"] for k in ("means", "inv_cov", "phase", "opac", "curv", "area")}
    grads = opre.activate_backward(act, w["means"], w["inv_cov"], np.zeros_like(raw["colours"]), w["phase"],
                                   w["opac"], w["curv"], w["area"])
    for key in opre.RAW_KEYS:
        ref = g[f"{mode}__grad_{key}"]
        if key == "colours":
            continue
        if np.linalg.norm(ref) == 0:
            assert np.linalg.norm(grads[key]) == 0, key
            continue
        assert rel_l2(grads[key], ref) < 2e-5, key


def test_oracle_isotropic_phase_matches_reference_torch_renderer(golden):
    """--phase_iso: field of the reference torch renderer (isotropic QPF) within 2e-6 (float32 vs float64)."""
    g = golden("torch_renderer_iso_rgb")
    W, H = int(g["W"]), int(g["H"])
    pl, ranges = osp.bin_lists(g["act_means"], W, H, osp.CULL_TORCH64_3SIGMA, radius3=g["act_radius3"])
    out = osp.splat_forward(g["act_means"], g["act_inv_cov"], g["colours"], g["act_phase"], g["act_opac"],
                            g["act_curv"], g["act_area"], g["act_k"], float(g["act_dxy2"]), W, H,
                            cull=osp.CULL_TORCH64_3SIGMA, point_list=pl, ranges=ranges, phase_iso=True)
    assert rel_l2(out, g["field"]) < 2e-6


def test_oracle_isotropic_adjoint_matches_finite_differences():
    rng = np.random.default_rng(8)
    n, W, H, C = 6, 20, 18, 3
    means = np.stack([rng.uniform(4, W - 4, n), rng.uniform(4, H - 4, n)], 1)
    inv = np.stack([rng.uniform(0.1, 0.3, n), rng.uniform(-0.05, 0.05, n), rng.uniform(0.1, 0.3, n)], 1)
    col, ph = rng.uniform(0, 1, (n, C)), rng.uniform(0, 6, (n, C))
    op, cv, ar = rng.uniform(0.3, 0.9, n), rng.normal(0, 3e4, n), rng.uniform(2, 6, n)
    k = 2 * np.pi / np.array([639e-9, 515e-9, 473e-9])
    dxy2 = 3.74e-6 ** 2
    G = rng.normal(size=(C, H, W)) + 1j * rng.normal(size=(C, H, W))
    args = [means, inv, col, ph, op, cv, ar]
    loss = lambda a: float(np.sum((osp.splat_forward(*a, k, dxy2, W, H, phase_iso=True) * np.conj(G)).real))
    grads = osp.splat_backward(G, *args, k, dxy2, W, H, phase_iso=True)
    for ai, (arr, gr) in enumerate(zip(args, grads)):
        for idx in [(0,) * arr.ndim, tuple(d - 1 for d in arr.shape)]:
            h = 1e-6 * max(1.0, abs(arr[idx]))
            ap = [a.copy() for a in args]
            am = [a.copy() for a in args]
            ap[ai][idx] += h
            am[ai][idx] -= h
            fd = (loss(ap) - loss(am)) / (2 * h)
            assert abs(gr[idx] - fd) <= 1e-5 * max(1.0, abs(fd)), (ai, idx, gr[idx], fd)
    assert np.all(grads[6] == 0)  # the area does not enter the isotropic phase
