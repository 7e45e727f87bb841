"""The bracket-predictor network's tensor-core kernels against plain FP32 / FP64 arithmetic."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 384, 192), (512, 128, 1024)])
def test_gemm_bf16_tensor_cores(M, N, K):
    """C = A B^T on tcgen05 (BF16 operands, FP32 accumulation) equals the FP32 product of the
    same BF16 values to FP32 summation-order round-off; accumulate adds to C"""
    import torch
    from agama_b200 import _native
    g = torch.Generator(device="cpu").manual_seed(M + N + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    C = torch.full((M, N), 7.0, dtype=torch.float32, device="cuda")
    ref = A.float() @ B.float().T
    L = _native.lib()
    _native.check(L.agama_gemmBf16Device(M, N, K, _native.VP(A.data_ptr()), _native.VP(B.data_ptr()),
                                         _native.VP(C.data_ptr()), N, 0, None))
    torch.cuda.synchronize()
    scale = np.sqrt(K)
    assert torch.max(torch.abs(C - ref)).item() <= 1e-5 * scale
    _native.check(L.agama_gemmBf16Device(M, N, K, _native.VP(A.data_ptr()), _native.VP(B.data_ptr()),
                                         _native.VP(C.data_ptr()), N, 1, None))
    torch.cuda.synchronize()
    assert torch.max(torch.abs(C - 2 * ref)).item() <= 2e-5 * scale
