// The bracket-predictor network (6 -> 128 -> 128 -> 128 -> 3, SiLU) and its tensor-core GEMM.
#pragma once
#include <cuda_runtime.h>

namespace agb {

/// C[M x N] (FP32, leading dimension ldc) = A[M x K] * B[N x K]^T (+ C), A and B BF16 row-major;
/// M, N multiples of 128, K a multiple of 64 (tcgen05 MMAs, mlp_gemm.cu)
void launchGemmBf16(int M, int N, int K, const void* A, const void* B, float* C, int ldc, bool accumulate,
    cudaStream_t stream);
/// throws if a GEMM launched since the process started gave up waiting for its tensor cores
void checkGemmError();

}  // namespace agb
