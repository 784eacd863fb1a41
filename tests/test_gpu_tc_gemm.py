"""The learned start's GEMM on the 5th-generation tensor cores (tcgen05.mma
kind::f16, operands staged by TMA with the 128 B swizzle, FP32 accumulation in
tensor memory) against a plain PyTorch FP32 reference of the same product.
The shapes cover the network's layers (n = 28 padded to 32, width 512 and
256), ragged row counts, K not a multiple of the 64-wide k-block, and N below
the 128-wide tile."""
import pytest

import closures_b200 as cb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(4096, 512, 512), (1000, 28, 512), (777, 512, 32), (130, 64, 200),
                                   (131072, 512, 512), (262144, 256, 256), (5, 32, 8)])
def test_tc_gemm_matches_fp32_reference(M, N, K):
    import torch
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn((M, K), device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn((N, K), device="cuda", generator=g).to(torch.bfloat16)
    C = cb.tc_gemm_bf16(A, B)
    ref = A.float() @ B.float().T
    # BF16 products are exact in FP32; only the summation order differs
    tol = 1e-5 * K * float(ref.abs().max())
    assert float((C - ref).abs().max()) <= tol
