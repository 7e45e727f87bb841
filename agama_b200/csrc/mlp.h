// The bracket-predictor network (6 -> 128 -> 128 -> 128 -> 3, SiLU) and its tensor-core GEMM.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "runtime.h"

namespace agb {

constexpr int MLP_INPUTS = 6, MLP_HIDDEN = 128, MLP_OUTPUTS = 3;
constexpr int MLP_NUM_PARAMS = MLP_HIDDEN * MLP_INPUTS + MLP_HIDDEN + 2 * (MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN) +
    MLP_OUTPUTS * MLP_HIDDEN + MLP_OUTPUTS;

struct MlpBatch;

/** The network on one device: FP32 parameters (W1 b1 W2 b2 W3 b3 W4 b4, weights [out][in]),
    Adam moments, BF16 copies of W2, W3 and their transposes for the tensor cores, and the input /
    output standardisation {x mean[6], x std[6], y mean[3], y std[3]}. */
struct Mlp {
    int device = 0;
    DevBuf<float> params, adamM, adamV, scaling;
    DevBuf<unsigned short> w2, w2T, w3, w3T;    // bfloat16 bit patterns
    DevBuf<int> error;
    long adamStep = 0;

    explicit Mlp(unsigned long long seed);
    /// re-derive the BF16 weight copies after the FP32 parameters changed
    void refreshWeights(cudaStream_t s);
    /// loss and gradient (NPARAM floats, device) of one batch of standardised inputs / targets /
    /// masks (device or host pointers); the batch size must be a multiple of 128
    float lossGradDevice(int B, const float* x, const float* t, const float* m, float* grad, cudaStream_t s);
    /// Adam training on n raw samples (standardisation derived from them); returns the mean loss
    /// of every epoch
    std::vector<float> train(long n, const float* x, const float* t, const float* m, int epochs, int batch,
        float lr, unsigned long long seed, cudaStream_t s);
    /// predictions (n x 3, raw units) for n raw inputs (n x 6), device pointers: the fused
    /// tensor-core inference kernel
    void predict(long n, const float* x, float* y, cudaStream_t s) const;
    /// throws if an inference kernel gave up waiting for its tensor cores
    void checkError() const;
private:
    void lossGrad(MlpBatch& bt, const float* maskSum, float* loss, float* grad, cudaStream_t s);
};

/// C[M x N] (FP32, leading dimension ldc) = A[M x K] * B[N x K]^T (+ C), A and B BF16 row-major;
/// M, N multiples of 128, K a multiple of 64 (tcgen05 MMAs, mlp_gemm.cu).  With a workspace
/// (workspaceFloats floats), outputs of few tiles are split over K across CTAs.
void launchGemmBf16(int M, int N, int K, const void* A, const void* B, float* C, int ldc, bool accumulate,
    cudaStream_t stream, float* workspace = nullptr, size_t workspaceFloats = 0);
/// set up the GEMM's per-device state (error flag, shared-memory limit) before a stream capture
void prepareGemm();
/// throws if a GEMM launched since the process started gave up waiting for its tensor cores
void checkGemmError();

}  // namespace agb
