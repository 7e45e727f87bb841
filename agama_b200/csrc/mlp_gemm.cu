// BF16 x BF16 -> FP32 GEMM on the fifth-generation tensor cores, the building block of the
// bracket-predictor network's training (umma.cuh: descriptors, tensor memory, MMA).
//
//   C[M x N] (FP32, row-major, leading dimension ldc) = A[M x K] * B[N x K]^T  (+ C if accumulate)
//
// A and B are BF16 row-major with K contiguous (both "K-major"), M and N multiples of 128, K a
// multiple of 64.  One CTA of 4 warps computes one 128 x 128 tile: K is walked in chunks of 64,
// each chunk staged into shared memory in the canonical layout and consumed by four 128x128x16
// MMAs issued by one thread into a 128-column tensor-memory accumulator; the accumulator is read
// back by all four warps (warp w owns rows 32w..32w+31).
#include "runtime.h"
#include "umma.cuh"
#include "mlp.h"
#include <cuda_bf16.h>
#include <map>
#include <mutex>

namespace agb {

namespace {

constexpr int GEMM_BM = 128, GEMM_BN = 128, GEMM_BK = 64;
constexpr int TILE_BYTES = GEMM_BM * GEMM_BK * 2;            // 16 KB per operand tile
constexpr int GEMM_STAGES = 2;
// two stages of (A, B) tiles, 64 KB, plus alignment: at most 3 CTAs (384 tensor-memory columns)
// on an SM, so an allocation never waits for another CTA's columns
constexpr int GEMM_SMEM = GEMM_STAGES * 2 * TILE_BYTES + 1024;
constexpr long MBAR_MAX_POLLS = 1L << 22;
constexpr int GEMM_MAX_SPLITS = 16;

/** One 128 x 128 tile of C = A B^T over this CTA's part of K (blockIdx.z of gridDim.z equal parts of
    Ksplit columns each; A and B rows have stride lda), written to C + blockIdx.z * splitStride.
    The K-chunks go through two shared-memory stages: the threads stage chunk j + 1 while the
    tensor cores run the MMAs of chunk j, and a stage is overwritten only after the mbarrier of the
    MMAs that read it has completed. */
__global__ void __launch_bounds__(128) gemmBf16Kernel(int Ksplit, int lda, const __nv_bfloat16* __restrict__ A,
    const __nv_bfloat16* __restrict__ B, float* __restrict__ C, int ldc, long splitStride, int accumulate,
    int* __restrict__ error)
{
    extern __shared__ unsigned char smemRaw[];
    __shared__ uint64_t mbar[GEMM_STAGES];
    __shared__ uint32_t tmemBase;
    unsigned char* tiles = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int bm = blockIdx.y * GEMM_BM, bn = blockIdx.x * GEMM_BN;
    const int kBegin = blockIdx.z * Ksplit, kEnd = kBegin + Ksplit;
    C += blockIdx.z * splitStride;

    if(warp == 0) umma::tmemAlloc(&tmemBase, 128);
    if(threadIdx.x == 0) for(int st = 0; st < GEMM_STAGES; st++) umma::mbarInit(&mbar[st], 1);
    umma::fenceBeforeSync();
    __syncthreads();
    umma::fenceAfterSync();
    const uint32_t tmem = tmemBase;
    constexpr uint32_t idesc = umma::instrDescBf16(GEMM_BM, GEMM_BN);
    constexpr uint32_t SBO = GEMM_BK / 8 * umma::CORE_BYTES;

    uint32_t parity[GEMM_STAGES] = { 0, 0 };
    bool ok = true;
    int chunk = 0;
    for(int k0 = kBegin; k0 < kEnd; k0 += GEMM_BK, chunk++) {
        const int st = chunk % GEMM_STAGES;
        unsigned char* tileA = tiles + st * 2 * TILE_BYTES;
        unsigned char* tileB = tileA + TILE_BYTES;
        if(chunk >= GEMM_STAGES) {
            // the MMAs of chunk - GEMM_STAGES read this stage: wait for them before overwriting it
            const bool done = umma::mbarWait(&mbar[st], parity[st], MBAR_MAX_POLLS);
            parity[st] ^= 1;
            ok = __syncthreads_and(done);
            if(!ok) break;
        }
        // stage the 128 x 64 chunks of A and B: 16-byte vectors = one row of one core matrix
        for(int v = threadIdx.x; v < GEMM_BM * GEMM_BK / 8; v += blockDim.x) {
            const int r = v / (GEMM_BK / 8), kc = v % (GEMM_BK / 8);
            const uint32_t off = umma::tileOffset(r, kc * 8, GEMM_BK);
            *reinterpret_cast<uint4*>(tileA + off) =
                *reinterpret_cast<const uint4*>(A + static_cast<size_t>(bm + r) * lda + k0 + kc * 8);
            *reinterpret_cast<uint4*>(tileB + off) =
                *reinterpret_cast<const uint4*>(B + static_cast<size_t>(bn + r) * lda + k0 + kc * 8);
        }
        umma::fenceSmemForAsync();
        __syncthreads();
        if(threadIdx.x == 0) {
            umma::fenceAfterSync();
            for(int kk = 0; kk < GEMM_BK / 16; kk++) {
                const uint64_t da = umma::smemDescriptor(umma::smemAddr(tileA) + kk * 2 * umma::LBO, umma::LBO, SBO);
                const uint64_t db = umma::smemDescriptor(umma::smemAddr(tileB) + kk * 2 * umma::LBO, umma::LBO, SBO);
                umma::mmaBf16(tmem, da, db, idesc, k0 > kBegin || kk > 0);
            }
            umma::commitTo(&mbar[st]);
        }
    }
    // the chunks whose completion has not been waited for yet (the last GEMM_STAGES), in order
    if(ok) {
        for(int j = chunk > GEMM_STAGES ? chunk - GEMM_STAGES : 0; j < chunk; j++) {
            const int st = j % GEMM_STAGES;
            const bool done = umma::mbarWait(&mbar[st], parity[st], MBAR_MAX_POLLS);
            parity[st] ^= 1;
            ok = __syncthreads_and(done);
            if(!ok) break;
        }
    }
    umma::fenceAfterSync();
    if(ok) {
        const int row = bm + warp * 32 + lane;
        for(int c0 = 0; c0 < GEMM_BN; c0 += 32) {
            float v[32];
            umma::tmemLoad32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + c0, v);
            float* out = C + static_cast<size_t>(row) * ldc + bn + c0;
#pragma unroll
            for(int j = 0; j < 32; j++) out[j] = accumulate ? out[j] + v[j] : v[j];
        }
    } else if(threadIdx.x == 0) {
        atomicExch(error, 1);
    }
    umma::fenceBeforeSync();
    __syncthreads();
    if(warp == 0) umma::tmemFree(tmem, 128);
}

/// C (+)= the sum of the split-K partial products, added in split order (deterministic)
__global__ void splitReduceKernel(int M, int N, int ldc, int splits, const float* __restrict__ part, float* __restrict__ C,
    int accumulate)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= M * N) return;
    const int r = i / N, c = i % N;
    float s = accumulate ? C[static_cast<size_t>(r) * ldc + c] : 0.f;
    for(int z = 0; z < splits; z++) s += part[static_cast<size_t>(z) * M * N + i];
    C[static_cast<size_t>(r) * ldc + c] = s;
}

/// per-device state of the GEMM: its completion-timeout flag (device memory of that device) and
/// whether the kernel's dynamic shared-memory limit has been raised there
struct GemmDeviceState {
    int* flag = nullptr;
    bool attr = false;
};
std::mutex g_gemmMutex;
std::map<int, GemmDeviceState> g_gemmState;

/// the state of the current device, set up on its first use (with that device current)
GemmDeviceState& gemmState()
{
    int dev;
    AGB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_gemmMutex);
    GemmDeviceState& st = g_gemmState[dev];        // map references stay valid as entries are added
    if(!st.flag) {
        AGB_CUDA(cudaMalloc(&st.flag, sizeof(int)));
        AGB_CUDA(cudaMemset(st.flag, 0, sizeof(int)));
    }
    if(!st.attr) {
        AGB_CUDA(cudaFuncSetAttribute(gemmBf16Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM));
        st.attr = true;
    }
    return st;
}

}  // namespace

void launchGemmBf16(int M, int N, int K, const void* A, const void* B, float* C, int ldc, bool accumulate,
    cudaStream_t stream, float* workspace, size_t workspaceFloats)
{
    if(M <= 0 || N <= 0 || K <= 0) return;
    if(M % GEMM_BM || N % GEMM_BN || K % GEMM_BK || ldc < N)
        throw std::invalid_argument("gemmBf16: M, N must be multiples of 128, K of 64, ldc >= N");
    GemmDeviceState& st = gemmState();
    // split K over several CTAs when the output has few tiles (the weight gradients: one 128 x 128
    // tile with K = batch): each split writes its partial tile to the workspace, then one kernel
    // sums them in order
    const int tiles = (M / GEMM_BM) * (N / GEMM_BN), chunks = K / GEMM_BK;
    int splits = 1;
    while(splits * 2 <= GEMM_MAX_SPLITS && tiles * splits * 2 <= 64 && chunks % (splits * 2) == 0 &&
          chunks / (splits * 2) >= 2 && workspace &&
          static_cast<size_t>(splits) * 2 * M * N <= workspaceFloats)
        splits *= 2;
    const dim3 grid(N / GEMM_BN, M / GEMM_BM, splits);
    if(splits == 1) {
        gemmBf16Kernel<<<grid, 128, GEMM_SMEM, stream>>>(K, K, static_cast<const __nv_bfloat16*>(A),
            static_cast<const __nv_bfloat16*>(B), C, ldc, 0, accumulate ? 1 : 0, st.flag);
    } else {
        gemmBf16Kernel<<<grid, 128, GEMM_SMEM, stream>>>(K / splits, K, static_cast<const __nv_bfloat16*>(A),
            static_cast<const __nv_bfloat16*>(B), workspace, N, static_cast<long>(M) * N, 0, st.flag);
        splitReduceKernel<<<(M * N + 255) / 256, 256, 0, stream>>>(M, N, ldc, splits, workspace, C, accumulate ? 1 : 0);
    }
    AGB_CUDA(cudaGetLastError());
}

void prepareGemm() { gemmState(); }

void checkGemmError()
{
    // the flag of the current device; cleared once read, so a timeout is reported once
    int* flag = gemmState().flag;
    int h = 0;
    AGB_CUDA(cudaMemcpy(&h, flag, sizeof(int), cudaMemcpyDeviceToHost));
    if(h) {
        AGB_CUDA(cudaMemset(flag, 0, sizeof(int)));
        throw std::runtime_error("gemmBf16: tensor-core completion barrier timed out");
    }
}

}  // namespace agb
