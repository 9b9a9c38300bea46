"""tcgen05 bf16 GEMM (mixed-precision building block) against a torch fp32
reference of the same product.  Tolerance: fp32 accumulation of exact bf16
products, 2e-5 of the largest |C| entry."""
import pytest
import torch

from afqmclab_b200 import capi

pytestmark = pytest.mark.gpu

TOL = 2e-5


def run(M, N, K, lda=None, ldb=None, splits=1, out_bf16=False, alpha=1.0, seed=0):
    g = torch.Generator(device="cuda").manual_seed(seed)
    lda = lda or K
    ldb = ldb or K
    A = torch.randn(M, lda, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, ldb, device="cuda", generator=g).to(torch.bfloat16)
    ldc = M
    dt = torch.bfloat16 if out_bf16 else torch.float32
    C = torch.full((splits, N, ldc), float("nan"), device="cuda", dtype=dt)
    capi.gemm_bf16_dev(M, N, K, A.data_ptr(), lda, B.data_ptr(), ldb, C.data_ptr(), ldc, out_bf16,
                       splits, N * ldc, alpha)
    ref = alpha * (A[:, :K].float() @ B[:, :K].float().T)
    got = C.float().sum(0).T
    return got, ref


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (128, 256, 128), (256, 512, 640),
                                   (200, 100, 130), (1000, 300, 200)])
def test_tc_gemm_matches_fp32(M, N, K):
    lda = (K + 7) // 8 * 8
    got, ref = run(M, N, K, lda=lda, ldb=lda)
    err = (got - ref).abs().max().item() / ref.abs().max().item()
    assert err < TOL, err


def test_tc_gemm_split_k():
    got, ref = run(1280, 512, 4096, splits=4)
    err = (got - ref).abs().max().item() / ref.abs().max().item()
    assert err < TOL, err


def test_tc_gemm_bf16_output_and_alpha():
    got, ref = run(256, 512, 640, out_bf16=True, alpha=0.25)
    err = (got - ref).abs().max().item() / ref.abs().max().item()
    assert err < 1e-2, err


# Large outputs take the persistent transposed kernel (at least one tile per
# SM): full tiles, ragged M / N / K edges, split K and bf16 output.
@pytest.mark.parametrize("M,N,K,splits", [(4096, 2048, 640, 1), (4100, 2000, 130, 1),
                                          (1280, 2048, 4096, 4), (16384, 256, 64, 1)])
def test_tc_gemm_persistent_matches_fp32(M, N, K, splits):
    lda = (K + 7) // 8 * 8
    got, ref = run(M, N, K, lda=lda, ldb=lda, splits=splits)
    err = (got - ref).abs().max().item() / ref.abs().max().item()
    assert err < TOL, err


def test_tc_gemm_persistent_bf16_output():
    got, ref = run(4096, 1024, 640, out_bf16=True, alpha=0.5)
    err = (got - ref).abs().max().item() / ref.abs().max().item()
    assert err < 1e-2, err
