"""GPU: the BF16 tcgen05 GEMM (cvqpg_gemm_bf16_tn) against float64 numpy.

BF16 x BF16 products are exact in FP32, so the only difference from the float64
reference is the FP32 accumulation order: gate 1e-5 relative L2 for the raw
product, 1e-5 for the FP32 epilogue outputs, and one BF16 rounding (2^-8
relative per element, gate 4e-3 relative L2) for the BF16 outputs.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _bf16(shape, seed, scale=1.0):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(shape, generator=g) * scale).to(torch.bfloat16)


def _ref(A, B):
    return A.double().numpy() @ B.double().numpy().T


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 384, 192), (128, 128, 1024), (384, 256, 576)])
def test_gemm_f32_matches_numpy(M, N, K):
    from complex_valued_quadratic_phase_gaussian_b200.mlp import gemm_bf16_tn
    A, B = _bf16((M, K), 1), _bf16((N, K), 2)
    C = torch.full((M, N), float("nan"), device="cuda")
    st = gemm_bf16_tn(A.cuda(), B.cuda(), out_f32=C)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    assert rel_l2(C.cpu().numpy(), _ref(A, B)) < 1e-5


def test_gemm_strided_operands_and_split_k():
    from complex_valued_quadratic_phase_gaussian_b200.mlp import gemm_bf16_tn
    M, N, K, splits = 256, 128, 1024, 4
    Abig, Bbig = _bf16((M, K + 64), 3), _bf16((N, K + 128), 4)
    A, B = Abig[:, 32:32 + K], Bbig[:, 64:64 + K]
    Ag, Bg = Abig.cuda()[:, 32:32 + K], Bbig.cuda()[:, 64:64 + K]
    slabs = torch.zeros((splits, M, N), device="cuda")
    st = gemm_bf16_tn(Ag, Bg, out_f32=slabs, splits=splits)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    assert rel_l2(slabs.sum(0).cpu().numpy(), _ref(A, B)) < 1e-5
    # each slab is its own K range
    ref0 = A[:, :K // splits].double().numpy() @ B[:, :K // splits].double().numpy().T
    assert rel_l2(slabs[0].cpu().numpy(), ref0) < 1e-5


def _gelu(z):
    from scipy.special import erf
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def _gelu_grad(z):
    from scipy.special import erf
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def test_gemm_bias_gelu_and_dgelu_epilogues():
    from complex_valued_quadratic_phase_gaussian_b200.mlp import (EPI_BIAS, EPI_BIAS_GELU, EPI_DGELU,
                                                                  gemm_bf16_tn)
    M, N, K, valid = 256, 256, 128, 200
    A, B = _bf16((M, K), 5, 0.2), _bf16((N, K), 6, 0.2)
    bias = torch.linspace(-0.5, 0.5, N)
    Z = torch.empty((M, N), device="cuda")
    H = torch.empty((M, N), dtype=torch.bfloat16, device="cuda")
    Ht = torch.empty((N, M), dtype=torch.bfloat16, device="cuda")
    st = gemm_bf16_tn(A.cuda(), B.cuda(), mode=EPI_BIAS_GELU, out_f32=Z, bias=bias.cuda(), out_bf16=H,
                      out_bf16_t=Ht, valid_n=valid)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    z_ref = _ref(A, B) + bias.double().numpy()[None]
    h_ref = _gelu(z_ref)
    h_ref[:, valid:] = 0.0
    assert rel_l2(Z.cpu().numpy(), z_ref) < 1e-5
    assert rel_l2(H.float().cpu().numpy(), h_ref) < 4e-3
    assert torch.equal(Ht.cpu(), H.cpu().T.contiguous())
    assert torch.count_nonzero(H[:, valid:]).item() == 0
    # plain bias epilogue
    Y = torch.empty((M, N), device="cuda")
    gemm_bf16_tn(A.cuda(), B.cuda(), mode=EPI_BIAS, out_f32=Y, bias=bias.cuda(), status=st)
    torch.cuda.synchronize()
    assert rel_l2(Y.cpu().numpy(), z_ref) < 1e-5
    # GELU derivative against the saved pre-activation
    G = torch.empty((M, N), dtype=torch.bfloat16, device="cuda")
    Gt = torch.empty((N, M), dtype=torch.bfloat16, device="cuda")
    gemm_bf16_tn(A.cuda(), B.cuda(), mode=EPI_DGELU, zin=Z, out_bf16=G, out_bf16_t=Gt, valid_n=valid, status=st)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    g_ref = _ref(A, B) * _gelu_grad(Z.double().cpu().numpy())
    g_ref[:, valid:] = 0.0
    assert rel_l2(G.float().cpu().numpy(), g_ref) < 4e-3
    assert torch.equal(Gt.cpu(), G.cpu().T.contiguous())


def test_bounded_wait_gives_up_and_reports():
    """The bounded mbarrier wait of the tcgen05 kernels: a barrier nothing arrives at makes it give
    up after its poll limit with status 4 and return; with an arrival it completes with status 0.
    The context stays usable (a GEMM runs right after)."""
    import ctypes
    from complex_valued_quadratic_phase_gaussian_b200 import _lib
    lib = _lib.lib()
    st = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    s = _lib.stream_of(torch.device("cuda"))
    _lib.check(lib.cvqpg_wait_probe(0, 4096, _lib.ptr(st), s), "cvqpg_wait_probe")
    torch.cuda.synchronize()
    assert int(st.item()) == 4
    _lib.check(lib.cvqpg_wait_probe(1, 4096, _lib.ptr(st), s), "cvqpg_wait_probe")
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    from complex_valued_quadratic_phase_gaussian_b200.mlp import gemm_bf16_tn
    A, B = _bf16((128, 64), 1), _bf16((128, 64), 2)
    C = torch.full((128, 128), float("nan"), device="cuda")
    gst = gemm_bf16_tn(A.cuda(), B.cuda(), out_f32=C)
    torch.cuda.synchronize()
    assert int(gst.item()) == 0
    assert rel_l2(C.cpu().numpy(), _ref(A, B)) < 1e-5
