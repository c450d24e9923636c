"""GPU: the allocation-free render entry point against the workspace one.

cvqpg_render_forward_noalloc exists for callers that cannot allocate device
memory where they render (a host that owns every allocation and passes only its
own buffers, a process under a fixed memory budget, code that must not call
cudaMalloc because it synchronises the device). Its scratch is a fixed array
inside the library, shared by every call, so this test calls it twice in a row
(a larger scene, then a smaller one that reuses the array with the first call's
contents still in it) and checks each result against cvqpg_render_forward,
which takes its scratch from a caller workspace. This file is named to be
collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


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
    radii = np.ceil(5 * np.sqrt(0.5 * (c00 + c11) + np.sqrt((0.5 * (c00 - c11)) ** 2 + c01 ** 2))).astype(np.int32)
    arrs = [means, inv, rng.uniform(0, 1, (n, C)).astype(np.float32),
            rng.uniform(0, 2 * np.pi, (n, C)).astype(np.float32), rng.uniform(0.2, 0.9, n).astype(np.float32),
            rng.normal(0, 800, n).astype(np.float32), (s[:, 0] * s[:, 1]).astype(np.float32)]
    k = (2 * np.pi / np.array([639e-9, 515e-9, 473e-9][:C])).astype(np.float32)
    return [torch.from_numpy(a).cuda() for a in arrs], torch.from_numpy(radii).cuda(), torch.from_numpy(k).cuda()


def _outputs(C, H, W, cap, lists):
    return (torch.empty((C, H, W), dtype=torch.complex64, device="cuda"),
            torch.empty(cap, dtype=torch.int32, device="cuda"), torch.empty((lists, 2), dtype=torch.int32, device="cuda"),
            torch.zeros(2, dtype=torch.int32, device="cuda"))


def _run(which, ins, radii, k, n, W, H, C, cap):
    from complex_valued_quadratic_phase_gaussian_b200 import _lib
    lib = _lib.lib()
    P = _lib.ptr
    out, pl, ranges, cnt = _outputs(C, H, W, cap, lib.cvqpg_render_num_lists(0, W, H))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    common = [P(t) for t in ins] + [P(radii), P(k), ctypes.c_float(3.74e-6 ** 2), n, W, H, C,
                                    P(torch.view_as_real(out)), P(pl), cap, P(ranges), P(cnt)]
    if which == "noalloc":
        st = lib.cvqpg_render_forward_noalloc(*common, stream)
    else:
        ws = _lib.workspace(_lib.size_query(lib.cvqpg_render_workspace_size, n, W, H, cap), "cuda")
        st = lib.cvqpg_render_forward(*common, P(ws), ws.numel(), stream)
    assert st == 0, lib.cvqpg_status_string(st)
    torch.cuda.synchronize()
    total, over = cnt.tolist()
    assert over == 0
    return out.cpu().numpy(), pl[:total].cpu().numpy(), ranges.cpu().numpy()


def test_noalloc_matches_workspace_entry_point_twice():
    cases = [(12000, 320, 256, 3, 150000, 1), (3000, 200, 136, 1, 60000, 2)]
    for n, W, H, C, cap, seed in cases:
        ins, radii, k = _scene(n, W, H, C, seed)
        ref_out, ref_pl, ref_ranges = _run("workspace", ins, radii, k, n, W, H, C, cap)
        out, pl, ranges = _run("noalloc", ins, radii, k, n, W, H, C, cap)
        assert np.array_equal(pl, ref_pl)
        assert np.array_equal(ranges, ref_ranges)
        assert rel_l2(out, ref_out) < 1e-5


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from complex_valued_quadratic_phase_gaussian_b200 import _lib
    lib = _lib.lib()
    z = ctypes.c_void_p(0)
    st = lib.cvqpg_render_forward_noalloc(z, z, z, z, z, z, z, z, z, ctypes.c_float(1.0), 16385, 64, 64, 1, z, z,
                                          1000, z, z, z)
    assert st == 5  # CVQPG_ERR_UNSUPPORTED
    st = lib.cvqpg_render_forward_noalloc(z, z, z, z, z, z, z, z, z, ctypes.c_float(1.0), 100, 64, 64, 1, z, z,
                                          262145, z, z, z)
    assert st == 5
