"""GPU: bit-exact tile lists and matching field/gradients against the reference's own compiled
CUDA rasterizer (built from the reference sources into oracle/_ref by oracle/build_ref.py)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import splat as osp
from oracle.torch_port import load_reference_extension

pytestmark = pytest.mark.gpu
SPLAT_KEYS = ("means", "inv_cov", "colours", "phase", "opac", "curv", "area")


@pytest.fixture(scope="module")
def ref_ext():
    ext = load_reference_extension()
    if ext is None:
        pytest.skip("reference extension not built (oracle/build_ref.py needs the reference sources)")
    return ext


def _scene(n, W, H, C, seed):
    rng = np.random.default_rng(seed)
    means = np.stack([rng.uniform(-6, W + 6, n), rng.uniform(-6, H + 6, n)], 1).astype(np.float32)
    s = np.exp(rng.normal(np.log(2.0), 0.3, (n, 2))) + 0.1
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
    k = (2 * np.pi / np.array([639e-9, 515e-9, 473e-9][:C])).astype(np.float32)
    return [means, inv, col, ph, op, cv, ar], radii, k


@pytest.mark.parametrize("C,W,H,n", [(3, 200, 136, 3000), (1, 256, 256, 4096)])
def test_lists_field_and_gradients_vs_reference_cuda(ref_ext, C, W, H, n):
    import complex_valued_quadratic_phase_gaussian_b200 as pkg
    ins, radii, k = _scene(n, W, H, C, 11 + C)
    T = [torch.from_numpy(a).cuda() for a in ins]
    R = torch.from_numpy(radii).cuda()
    K = torch.from_numpy(k).cuda()
    dxy2 = float(np.float32(3.74e-6 ** 2))
    rr, ri, rpl, rranges = ref_ext.qpf_render_forward(*T, R, K, dxy2, W, H, C)
    mr, mi, mpl, mranges = pkg.ext().qpf_render_forward(*T, R, K, dxy2, W, H, C)
    assert torch.equal(rpl.cpu(), mpl.cpu()), "per-tile Gaussian lists differ"
    assert torch.equal(rranges.cpu(), mranges.cpu()), "tile ranges differ"
    ref_field = rr.cpu().numpy() + 1j * ri.cpu().numpy()
    got = mr.cpu().numpy() + 1j * mi.cpu().numpy()
    assert rel_l2(got, ref_field) < 1e-5  # the reference uses __sincosf; both are float32
    rng = np.random.default_rng(3)
    gr = torch.from_numpy(rng.normal(size=(C, H, W)).astype(np.float32)).cuda()
    gi = torch.from_numpy(rng.normal(size=(C, H, W)).astype(np.float32)).cuda()
    dref = ref_ext.qpf_render_backward(gr, gi, *T, K, rpl, rranges, dxy2, W, H, C)
    dgot = pkg.ext().qpf_render_backward(gr, gi, *T, K, mpl, mranges, dxy2, W, H, C)
    for key, a, b in zip(SPLAT_KEYS, dgot, dref):
        assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-4, key
