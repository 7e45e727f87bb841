// The bracket-predictor network: 6 -> 128 -> 128 -> 128 -> 3 with SiLU, BF16 weights and
// activations in the two 128 x 128 layers (FP32 accumulation on the tensor cores), FP32 master
// parameters and Adam.  Training: forward and backward passes over a batch with the tcgen05 GEMM
// of mlp_gemm.cu for every 128 x 128 product (forward activations, input gradients, weight
// gradients); the 6-wide first and 3-wide last layers, biases, activations and the optimiser are
// small elementwise / reduction kernels.  Inference: one fused kernel per 128 points that keeps
// both hidden products in tensor memory and shared memory (mlpInferKernel).
//
// Parameter vector (FP32, row-major weights [out][in]): W1[128x6] b1 W2[128x128] b2 W3[128x128] b3
// W4[3x128] b4.
#include "runtime.h"
#include "umma.cuh"
#include "mlp.h"
#include "host_pipeline.h"
#include <cuda_bf16.h>
#include <random>
#include <mutex>
#include <set>
#include <algorithm>
#include <cmath>

namespace agb {

namespace {

constexpr int H = MLP_HIDDEN, NIN = MLP_INPUTS, NOUT = MLP_OUTPUTS;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + H * NIN, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
    OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + H * H, OFF_W4 = OFF_B3 + H, OFF_B4 = OFF_W4 + NOUT * H,
    NPARAM = OFF_B4 + NOUT;
static_assert(NPARAM == MLP_NUM_PARAMS, "parameter layout");

/// SiLU z sigma(z) and its derivative, with the fast exponential and division of the special
/// function unit (relative error ~1e-6: far below the BF16 rounding of the activations)
__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) { const float s = __fdividef(1.f, 1.f + __expf(-z)); return s * (1.f + z * (1.f - s)); }

// ---------------------------------------------------------------- elementwise training kernels

/// z1 = x W1^T + b1 (x already standardised), h1 = silu(z1) in BF16, also transposed [128 x B]
__global__ void layer1Kernel(int B, const float* __restrict__ x, const float* __restrict__ p, float* __restrict__ z,
    __nv_bfloat16* __restrict__ hb, __nv_bfloat16* __restrict__ hbT)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if(idx >= B * H) return;
    const int b = idx / H, c = idx % H;
    float s = p[OFF_B1 + c];
    for(int k = 0; k < NIN; k++) s += x[b * NIN + k] * p[OFF_W1 + c * NIN + k];
    z[idx] = s;
    const __nv_bfloat16 v = __float2bfloat16_rn(silu(s));
    hb[idx] = v;
    hbT[static_cast<size_t>(c) * B + b] = v;
}

/// z = (GEMM output) + bias, h = silu(z): BF16 copies (row-major and transposed) and optionally FP32
__global__ void biasActKernel(int B, float* __restrict__ z, const float* __restrict__ bias,
    __nv_bfloat16* __restrict__ hb, __nv_bfloat16* __restrict__ hbT, float* __restrict__ hf)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if(idx >= B * H) return;
    const int b = idx / H, c = idx % H;
    const float s = z[idx] + bias[c];
    z[idx] = s;
    const float h = silu(s);
    if(hf) hf[idx] = h;
    if(hb) {
        const __nv_bfloat16 v = __float2bfloat16_rn(h);
        hb[idx] = v;
        hbT[static_cast<size_t>(c) * B + b] = v;
    }
}

/// y = h3 W4^T + b4; loss terms and dy = 2 m (y - t) / S
__global__ void outputLossKernel(int B, const float* __restrict__ h3, const float* __restrict__ p,
    const float* __restrict__ t, const float* __restrict__ m, const float* __restrict__ maskSum, float* __restrict__ dy,
    float* __restrict__ loss)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if(idx >= B * NOUT) return;
    const float invS = 1.f / fmaxf(*maskSum, 1.f);
    const int b = idx / NOUT, j = idx % NOUT;
    float s = p[OFF_B4 + j];
    for(int c = 0; c < H; c++) s += h3[static_cast<size_t>(b) * H + c] * p[OFF_W4 + j * H + c];
    const float d = s - t[idx];
    dy[idx] = 2.f * m[idx] * d * invS;
    atomicAdd(loss, m[idx] * d * d * invS);
}

/// dz3 = (dy W4) * silu'(z3), in BF16 (row-major and transposed) and FP32
__global__ void backOutputKernel(int B, const float* __restrict__ dy, const float* __restrict__ p,
    const float* __restrict__ z, float* __restrict__ dz, __nv_bfloat16* __restrict__ dzb, __nv_bfloat16* __restrict__ dzbT)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if(idx >= B * H) return;
    const int b = idx / H, c = idx % H;
    float s = 0;
    for(int j = 0; j < NOUT; j++) s += dy[b * NOUT + j] * p[OFF_W4 + j * H + c];
    const float d = s * dsilu(z[idx]);
    dz[idx] = d;
    const __nv_bfloat16 v = __float2bfloat16_rn(d);
    dzb[idx] = v;
    dzbT[static_cast<size_t>(c) * B + b] = v;
}

/// dz = (GEMM output dh) * silu'(z) in place, plus BF16 copies
__global__ void backActKernel(int B, float* __restrict__ dh, const float* __restrict__ z,
    __nv_bfloat16* __restrict__ dzb, __nv_bfloat16* __restrict__ dzbT)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if(idx >= B * H) return;
    const int b = idx / H, c = idx % H;
    const float d = dh[idx] * dsilu(z[idx]);
    dh[idx] = d;
    if(dzb) {
        const __nv_bfloat16 v = __float2bfloat16_rn(d);
        dzb[idx] = v;
        dzbT[static_cast<size_t>(c) * B + b] = v;
    }
}

/// gradients of the small layers and of all biases: one block per output unit, reduction over B
///   role 0: dW4 row j and db4 (from dy, h3); role 1: db of a hidden layer (from dz);
///   role 2: dW1 row c and db1 (from dz1, x)
__global__ void reduceGradKernel(int B, int role, const float* __restrict__ a, const float* __restrict__ bsrc,
    float* __restrict__ grad, int offW, int offB)
{
    __shared__ float red[NIN + 1][256];
    const int unit = blockIdx.x;
    float acc[NIN + 1] = {};
    for(int b = threadIdx.x; b < B; b += blockDim.x) {
        if(role == 0) {            // a = dy [B x 3], bsrc = h3 [B x 128]; unit = column c of dW4 (all j)
            for(int j = 0; j < NOUT; j++) acc[j] += a[b * NOUT + j] * bsrc[static_cast<size_t>(b) * H + unit];
        } else if(role == 1) {     // a = dz [B x 128]
            acc[0] += a[static_cast<size_t>(b) * H + unit];
        } else {                   // a = dz1 [B x 128], bsrc = x [B x 6]
            const float d = a[static_cast<size_t>(b) * H + unit];
            for(int k = 0; k < NIN; k++) acc[k] += d * bsrc[b * NIN + k];
            acc[NIN] += d;
        }
    }
    for(int k = 0; k <= NIN; k++) red[k][threadIdx.x] = acc[k];
    __syncthreads();
    for(int s = blockDim.x / 2; s > 0; s >>= 1) {
        if(threadIdx.x < s)
            for(int k = 0; k <= NIN; k++) red[k][threadIdx.x] += red[k][threadIdx.x + s];
        __syncthreads();
    }
    if(threadIdx.x != 0) return;
    if(role == 0) {
        for(int j = 0; j < NOUT; j++) grad[offW + j * H + unit] = red[j][0];
    } else if(role == 1) {
        grad[offB + unit] = red[0][0];
    } else {
        for(int k = 0; k < NIN; k++) grad[offW + unit * NIN + k] = red[k][0];
        grad[offB + unit] = red[NIN][0];
    }
}

/// db4 = sum over the batch of dy
__global__ void outputBiasGradKernel(int B, const float* __restrict__ dy, float* __restrict__ grad)
{
    __shared__ float red[NOUT][256];
    float acc[NOUT] = {};
    for(int b = threadIdx.x; b < B; b += blockDim.x)
        for(int j = 0; j < NOUT; j++) acc[j] += dy[b * NOUT + j];
    for(int j = 0; j < NOUT; j++) red[j][threadIdx.x] = acc[j];
    __syncthreads();
    for(int s = blockDim.x / 2; s > 0; s >>= 1) {
        if(threadIdx.x < s) for(int j = 0; j < NOUT; j++) red[j][threadIdx.x] += red[j][threadIdx.x + s];
        __syncthreads();
    }
    if(threadIdx.x == 0) for(int j = 0; j < NOUT; j++) grad[OFF_B4 + j] = red[j][0];
}

/// BF16 copies of W2, W3 (as [out][in]) and their transposes ([in][out])
__global__ void weightCopiesKernel(const float* __restrict__ p, __nv_bfloat16* __restrict__ w2, __nv_bfloat16* __restrict__ w2T,
    __nv_bfloat16* __restrict__ w3, __nv_bfloat16* __restrict__ w3T)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if(idx >= H * H) return;
    const int o = idx / H, i = idx % H;
    w2[idx] = __float2bfloat16_rn(p[OFF_W2 + idx]);
    w2T[i * H + o] = w2[idx];
    w3[idx] = __float2bfloat16_rn(p[OFF_W3 + idx]);
    w3T[i * H + o] = w3[idx];
}

/// standardise: x' = (x - mean) / std per column
__global__ void standardiseKernel(long n, int ncol, const float* __restrict__ in, const float* __restrict__ mean,
    const float* __restrict__ stdv, float* __restrict__ out)
{
    const long idx = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if(idx >= n * ncol) return;
    const int c = static_cast<int>(idx % ncol);
    out[idx] = (in[idx] - mean[c]) / stdv[c];
}

/// device-side state of a training run, advanced by the kernels of each step, so that a step
/// replays from a CUDA graph without the host: the batch of the epoch's permutation, the Adam step
/// count, the batch's mask sum, the learning rate of the epoch and the loss sums
struct TrainState {
    int batchIndex;
    int adamStep;
    float maskSum;
    float lr;
    float loss;
    float lossSum;
};

/// the batch's rows by the epoch's permutation (x: NIN, t and m: NOUT columns) and the sum of its
/// masks (the loss normalisation)
__global__ void gatherBatchKernel(int B, const int* __restrict__ perm, TrainState* __restrict__ st,
    const float* __restrict__ xs, const float* __restrict__ ts, const float* __restrict__ ms,
    float* __restrict__ x, float* __restrict__ t, float* __restrict__ m)
{
    __shared__ float red[256];
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    float msum = 0;
    if(b < B) {
        const size_t row = static_cast<size_t>(perm[static_cast<size_t>(st->batchIndex) * B + b]);
        for(int k = 0; k < NIN; k++) x[b * NIN + k] = xs[row * NIN + k];
        for(int j = 0; j < NOUT; j++) {
            t[b * NOUT + j] = ts[row * NOUT + j];
            const float mv = ms[row * NOUT + j];
            m[b * NOUT + j] = mv;
            msum += mv;
        }
    }
    red[threadIdx.x] = msum;
    __syncthreads();
    for(int s2 = blockDim.x / 2; s2 > 0; s2 >>= 1) {
        if(threadIdx.x < s2) red[threadIdx.x] += red[threadIdx.x + s2];
        __syncthreads();
    }
    if(threadIdx.x == 0) atomicAdd(&st->maskSum, red[0]);      // integer-valued: exact in any order
}

/// the end of a step: loss into the epoch's sum, counters advanced, the mask sum cleared
__global__ void finishStepKernel(TrainState* st)
{
    st->lossSum += st->loss;
    st->loss = 0;
    st->maskSum = 0;
    st->batchIndex++;
    st->adamStep++;
}

/// the start of an epoch: learning rate, batch counter and loss sum
__global__ void startEpochKernel(TrainState* st, float lr)
{
    st->lr = lr;
    st->batchIndex = 0;
    st->lossSum = 0;
    st->loss = 0;
    st->maskSum = 0;
}

/// Adam (Kingma & Ba 2015) on the FP32 parameters; the step count and learning rate come from the
/// training state (bias corrections 1 - beta^t for the step t = adamStep + 1)
__global__ void adamKernel(int np, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
    float* __restrict__ v, const TrainState* __restrict__ st, float beta1, float beta2, float eps)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= np) return;
    const float step = static_cast<float>(st->adamStep + 1), lr = st->lr;
    const float c1 = 1 - powf(beta1, step), c2 = 1 - powf(beta2, step);
    const float gi = g[i];
    m[i] = beta1 * m[i] + (1 - beta1) * gi;
    v[i] = beta2 * v[i] + (1 - beta2) * gi * gi;
    p[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}


// ---------------------------------------------------------------- fused inference

constexpr int INF_SMEM = 3 * H * H * 2 + 2048;         // W2, W3, activation tile (BF16) + alignment
constexpr long INF_MAX_POLLS = 1L << 22;

/// SiLU of the inference kernel: z sigmoid(z) = z/2 (1 + tanh(z/2)) with the single-instruction
/// hardware tanh approximation (relative error ~2^-11, below the BF16 rounding that follows)
__device__ __forceinline__ float siluFast(float z)
{
    const float hz = 0.5f * z;
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(hz));
    return fmaf(hz, t, hz);
}

// threads per point (row of a tile): 1, 2 or 4; on B200, 1e6 points took 0.214, 0.218, 0.236 ms
constexpr int INF_ROW_THREADS = 1;
constexpr int INF_THREADS = 128 * INF_ROW_THREADS, INF_COLS = H / INF_ROW_THREADS;

/** Forward pass of 128 points per CTA iteration, persistent over tiles, INF_ROW_THREADS threads
    per point: thread t owns row t % 128 of the tile and the INF_COLS columns starting at
    INF_COLS (t / 128) (the tensor-memory rows of a warp are those of its warp index modulo 4).  Layer 1 on the FP32 pipe, the
    two 128 x 128 layers as tcgen05 MMAs (A = the tile's BF16 activations, B = the BF16 weights,
    both staged in shared memory in the canonical K-major layout, accumulator in 128 tensor-memory
    columns), SiLU epilogues from tensor-memory loads, layer 4 fused into the last epilogue (the
    threads of a row add their partial outputs through shared memory). */
__global__ void __launch_bounds__(INF_THREADS, 2) mlpInferKernel(long n, const float* __restrict__ xin,
    float* __restrict__ yout, const float* __restrict__ p, const __nv_bfloat16* __restrict__ w2,
    const __nv_bfloat16* __restrict__ w3, const float* __restrict__ scale, int* __restrict__ error)
{
    extern __shared__ unsigned char smemRaw[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmemBase;
    __shared__ __align__(16) float sW1T[NIN][H];            // layer-1 weights, transposed
    __shared__ __align__(16) float sW4T[H][4];               // layer-4 weights [unit][output], padded
    __shared__ __align__(16) float sB1[H], sB2[H], sB3[H];
    __shared__ float sB4[NOUT], sScale[2 * NIN + 2 * NOUT];
    __shared__ float sPart[INF_ROW_THREADS > 1 ? INF_ROW_THREADS - 1 : 1][NOUT][128];  // partial layer-4 sums
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
    unsigned char* tW2 = base;
    unsigned char* tW3 = base + H * H * 2;
    unsigned char* tA = base + 2 * H * H * 2;
    const int tid = threadIdx.x, warp = tid / 32, row = tid % 128, half = tid / 128;   // half: the row's column block
    const int cBegin = half * INF_COLS;

    for(int k = tid; k < H * NIN; k += INF_THREADS) sW1T[k % NIN][k / NIN] = p[OFF_W1 + k];
    for(int k = tid; k < H * 4; k += INF_THREADS) sW4T[k / 4][k % 4] = k % 4 < NOUT ? p[OFF_W4 + (k % 4) * H + k / 4] : 0.f;
    for(int k = tid; k < H; k += INF_THREADS) { sB1[k] = p[OFF_B1 + k]; sB2[k] = p[OFF_B2 + k]; sB3[k] = p[OFF_B3 + k]; }
    if(tid < NOUT) sB4[tid] = p[OFF_B4 + tid];
    if(tid < 2 * NIN + 2 * NOUT) sScale[tid] = scale[tid];
    // weights into the canonical layout: row o (output unit) = MMA "B" row, K = input unit
    for(int v = tid; v < H * H / 8; v += INF_THREADS) {
        const int r = v / (H / 8), kc = v % (H / 8);
        const uint32_t off = umma::tileOffset(r, kc * 8, H);
        *reinterpret_cast<uint4*>(tW2 + off) = *reinterpret_cast<const uint4*>(w2 + r * H + kc * 8);
        *reinterpret_cast<uint4*>(tW3 + off) = *reinterpret_cast<const uint4*>(w3 + r * H + kc * 8);
    }
    if(warp == 0) umma::tmemAlloc(&tmemBase, 128);
    if(tid == 0) umma::mbarInit(&mbar, 1);
    umma::fenceBeforeSync();
    __syncthreads();
    umma::fenceAfterSync();
    const uint32_t tmem = tmemBase;
    const uint32_t tmemRow = tmem + (static_cast<uint32_t>((warp % 4) * 32) << 16);
    constexpr uint32_t idesc = umma::instrDescBf16(128, H);
    constexpr uint32_t SBO = H / 8 * umma::CORE_BYTES;
    uint32_t parity = 0;
    bool ok = true;

    // write 32 activations of this thread's row (columns c0..c0+31) as BF16 in the canonical layout
    auto storeRow = [&](const float* h, int c0) {
#pragma unroll
        for(int q = 0; q < 4; q++) {
            uint4 v;
            __nv_bfloat162 p2[4];
#pragma unroll
            for(int e = 0; e < 4; e++) p2[e] = __floats2bfloat162_rn(h[q * 8 + 2 * e], h[q * 8 + 2 * e + 1]);
            v.x = *reinterpret_cast<uint32_t*>(&p2[0]); v.y = *reinterpret_cast<uint32_t*>(&p2[1]);
            v.z = *reinterpret_cast<uint32_t*>(&p2[2]); v.w = *reinterpret_cast<uint32_t*>(&p2[3]);
            *reinterpret_cast<uint4*>(tA + umma::tileOffset(row, c0 + q * 8, H)) = v;
        }
    };
    auto runLayer = [&](unsigned char* tW) {
        umma::fenceSmemForAsync();
        __syncthreads();
        if(tid == 0) {
            umma::fenceAfterSync();
            for(int kk = 0; kk < H / 16; kk++)
                umma::mmaBf16(tmem, umma::smemDescriptor(umma::smemAddr(tA) + kk * 2 * umma::LBO, umma::LBO, SBO),
                    umma::smemDescriptor(umma::smemAddr(tW) + kk * 2 * umma::LBO, umma::LBO, SBO), idesc, kk > 0);
            umma::commitTo(&mbar);
        }
        const bool done = umma::mbarWait(&mbar, parity, INF_MAX_POLLS);
        parity ^= 1;
        ok = __syncthreads_and(done);
        umma::fenceAfterSync();
    };

    const long tiles = (n + 127) / 128;
    for(long tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const long i = tile * 128 + row;
        const bool valid = i < n;
        float x[NIN];
        for(int k = 0; k < NIN; k++) x[k] = valid ? (xin[i * NIN + k] - sScale[k]) / sScale[NIN + k] : 0.f;
        for(int c0 = cBegin; c0 < cBegin + INF_COLS; c0 += 32) {
            float h[32];
#pragma unroll
            for(int c = 0; c < 32; c += 4) {
                float4 acc = *reinterpret_cast<const float4*>(&sB1[c0 + c]);
#pragma unroll
                for(int k = 0; k < NIN; k++) {
                    const float4 w = *reinterpret_cast<const float4*>(&sW1T[k][c0 + c]);
                    acc.x += x[k] * w.x; acc.y += x[k] * w.y; acc.z += x[k] * w.z; acc.w += x[k] * w.w;
                }
                h[c] = siluFast(acc.x); h[c + 1] = siluFast(acc.y); h[c + 2] = siluFast(acc.z); h[c + 3] = siluFast(acc.w);
            }
            storeRow(h, c0);
        }
        runLayer(tW2);
        if(!ok) break;
        for(int c0 = cBegin; c0 < cBegin + INF_COLS; c0 += 32) {
            float h[32];
            umma::tmemLoad32(tmemRow + c0, h);
#pragma unroll
            for(int c = 0; c < 32; c += 4) {
                const float4 b = *reinterpret_cast<const float4*>(&sB2[c0 + c]);
                h[c] = siluFast(h[c] + b.x); h[c + 1] = siluFast(h[c + 1] + b.y);
                h[c + 2] = siluFast(h[c + 2] + b.z); h[c + 3] = siluFast(h[c + 3] + b.w);
            }
            storeRow(h, c0);
        }
        umma::fenceBeforeSync();
        runLayer(tW3);
        if(!ok) break;
        float y[NOUT];
        for(int j = 0; j < NOUT; j++) y[j] = half == 0 ? sB4[j] : 0.f;
        for(int c0 = cBegin; c0 < cBegin + INF_COLS; c0 += 32) {
            float h[32];
            umma::tmemLoad32(tmemRow + c0, h);
#pragma unroll
            for(int c = 0; c < 32; c++) {
                const float a = siluFast(h[c] + sB3[c0 + c]);
                const float4 w = *reinterpret_cast<const float4*>(&sW4T[c0 + c][0]);
                y[0] += a * w.x; y[1] += a * w.y; y[2] += a * w.z;
            }
        }
        if(half > 0)
            for(int j = 0; j < NOUT; j++) sPart[half - 1][j][row] = y[j];
        umma::fenceBeforeSync();
        __syncthreads();        // the partial sums are in place; the tile's activations may be rewritten
        if(half == 0 && valid)
            for(int j = 0; j < NOUT; j++) {
                float v = y[j];
                for(int q = 0; q < INF_ROW_THREADS - 1; q++) v += sPart[q][j][row];
                yout[i * NOUT + j] = v * sScale[2 * NIN + NOUT + j] + sScale[2 * NIN + j];
            }
    }
    if(!ok && tid == 0) atomicExch(error, 1);
    umma::fenceBeforeSync();
    __syncthreads();
    if(warp == 0) umma::tmemFree(tmem, 128);
}

}  // namespace

// ---------------------------------------------------------------- host side

Mlp::Mlp(unsigned long long seed)
{
    std::vector<float> h(NPARAM, 0.f);
    std::mt19937_64 rng(seed);
    auto init = [&](int off, int out, int in) {
        std::normal_distribution<float> nd(0.f, std::sqrt(2.f / in));     // He initialisation
        for(int k = 0; k < out * in; k++) h[off + k] = nd(rng);
    };
    init(OFF_W1, H, NIN); init(OFF_W2, H, H); init(OFF_W3, H, H); init(OFF_W4, NOUT, H);
    for(int k = OFF_W4; k < OFF_W4 + NOUT * H; k++) h[k] *= 0.1f;
    AGB_CUDA(cudaGetDevice(&device));
    params.upload(h);
    std::vector<float> zeros(NPARAM, 0.f);
    adamM.upload(zeros);
    adamV.upload(zeros);
    std::vector<float> sc(2 * NIN + 2 * NOUT, 0.f);
    for(int k = 0; k < NIN; k++) sc[NIN + k] = 1.f;
    for(int k = 0; k < NOUT; k++) sc[2 * NIN + NOUT + k] = 1.f;
    scaling.upload(sc);
    w2.alloc(H * H); w2T.alloc(H * H); w3.alloc(H * H); w3T.alloc(H * H);
    error.alloc(1);
    AGB_CUDA(cudaMemset(error.ptr, 0, sizeof(int)));
    refreshWeights(0);
}

void Mlp::refreshWeights(cudaStream_t s)
{
    weightCopiesKernel<<<(H * H + 255) / 256, 256, 0, s>>>(params.ptr, reinterpret_cast<__nv_bfloat16*>(w2.ptr),
        reinterpret_cast<__nv_bfloat16*>(w2T.ptr), reinterpret_cast<__nv_bfloat16*>(w3.ptr),
        reinterpret_cast<__nv_bfloat16*>(w3T.ptr));
    AGB_CUDA(cudaGetLastError());
}

/// the per-batch work buffers of the training pass (B rows)
struct MlpBatch {
    int B;
    float *x, *t, *m, *z1, *z2, *z3, *h3, *dy, *dh, *loss, *maskSum, *ws;
    __nv_bfloat16 *h1b, *h1bT, *h2b, *h2bT, *dzb, *dzbT;
    static constexpr size_t WS_FLOATS = 16 * H * H;      // split-K partial tiles of the weight gradients
    Scratch mem;
    MlpBatch(int b, cudaStream_t s) : B(b), mem(bytes(b), s) {
        char* q = static_cast<char*>(mem.ptr);
        auto take = [&](size_t n) { char* r = q; q += (n + 255) / 256 * 256; return r; };
        ws = reinterpret_cast<float*>(take(WS_FLOATS * 4));
        maskSum = reinterpret_cast<float*>(take(4));
        x = reinterpret_cast<float*>(take(B * NIN * 4)); t = reinterpret_cast<float*>(take(B * NOUT * 4));
        m = reinterpret_cast<float*>(take(B * NOUT * 4));
        z1 = reinterpret_cast<float*>(take(B * H * 4)); z2 = reinterpret_cast<float*>(take(B * H * 4));
        z3 = reinterpret_cast<float*>(take(B * H * 4)); h3 = reinterpret_cast<float*>(take(B * H * 4));
        dy = reinterpret_cast<float*>(take(B * NOUT * 4)); dh = reinterpret_cast<float*>(take(B * H * 4));
        loss = reinterpret_cast<float*>(take(4));
        h1b = reinterpret_cast<__nv_bfloat16*>(take(B * H * 2)); h1bT = reinterpret_cast<__nv_bfloat16*>(take(B * H * 2));
        h2b = reinterpret_cast<__nv_bfloat16*>(take(B * H * 2)); h2bT = reinterpret_cast<__nv_bfloat16*>(take(B * H * 2));
        dzb = reinterpret_cast<__nv_bfloat16*>(take(B * H * 2)); dzbT = reinterpret_cast<__nv_bfloat16*>(take(B * H * 2));
    }
    static size_t bytes(int B) {
        return static_cast<size_t>(B) * (NIN * 4 + 3 * NOUT * 4 + 5 * H * 4 + 6 * H * 2) + WS_FLOATS * 4 + 19 * 256;
    }
};

namespace {
inline int blocks(long n, int b) { return static_cast<int>((n + b - 1) / b); }
}

/// loss and gradient of one batch already in bt.x / bt.t / bt.m (standardised); grad: NPARAM
/// floats; the loss is normalised by the mask sum at maskSum and added to loss (device pointers)
void Mlp::lossGrad(MlpBatch& bt, const float* maskSum, float* loss, float* grad, cudaStream_t s)
{
    const int B = bt.B;
    // forward
    layer1Kernel<<<blocks(B * H, 256), 256, 0, s>>>(B, bt.x, params.ptr, bt.z1, bt.h1b, bt.h1bT);
    launchGemmBf16(B, H, H, bt.h1b, w2.ptr, bt.z2, H, false, s);
    biasActKernel<<<blocks(B * H, 256), 256, 0, s>>>(B, bt.z2, params.ptr + OFF_B2, bt.h2b, bt.h2bT, nullptr);
    launchGemmBf16(B, H, H, bt.h2b, w3.ptr, bt.z3, H, false, s);
    biasActKernel<<<blocks(B * H, 256), 256, 0, s>>>(B, bt.z3, params.ptr + OFF_B3, nullptr, nullptr, bt.h3);
    outputLossKernel<<<blocks(B * NOUT, 256), 256, 0, s>>>(B, bt.h3, params.ptr, bt.t, bt.m, maskSum, bt.dy, loss);
    // backward: output layer
    reduceGradKernel<<<H, 256, 0, s>>>(B, 0, bt.dy, bt.h3, grad, OFF_W4, 0);
    outputBiasGradKernel<<<1, 256, 0, s>>>(B, bt.dy, grad);
    backOutputKernel<<<blocks(B * H, 256), 256, 0, s>>>(B, bt.dy, params.ptr, bt.z3, bt.dh, bt.dzb, bt.dzbT);
    // layer 3: dW3 = dz3^T h2, db3, dh2 = dz3 W3
    launchGemmBf16(H, H, B, bt.dzbT, bt.h2bT, grad + OFF_W3, H, false, s, bt.ws, MlpBatch::WS_FLOATS);
    reduceGradKernel<<<H, 256, 0, s>>>(B, 1, bt.dh, nullptr, grad, 0, OFF_B3);
    launchGemmBf16(B, H, H, bt.dzb, w3T.ptr, bt.dh, H, false, s);
    backActKernel<<<blocks(B * H, 256), 256, 0, s>>>(B, bt.dh, bt.z2, bt.dzb, bt.dzbT);
    // layer 2: dW2 = dz2^T h1, db2, dh1 = dz2 W2
    launchGemmBf16(H, H, B, bt.dzbT, bt.h1bT, grad + OFF_W2, H, false, s, bt.ws, MlpBatch::WS_FLOATS);
    reduceGradKernel<<<H, 256, 0, s>>>(B, 1, bt.dh, nullptr, grad, 0, OFF_B2);
    launchGemmBf16(B, H, H, bt.dzb, w2T.ptr, bt.dh, H, false, s);
    backActKernel<<<blocks(B * H, 256), 256, 0, s>>>(B, bt.dh, bt.z1, nullptr, nullptr);
    // layer 1
    reduceGradKernel<<<H, 256, 0, s>>>(B, 2, bt.dh, bt.x, grad, OFF_W1, OFF_B1);
    AGB_CUDA(cudaGetLastError());
}

float Mlp::lossGradDevice(int B, const float* x, const float* t, const float* m, float* grad, cudaStream_t s)
{
    if(B <= 0 || B % 128) throw std::invalid_argument("mlp: the batch size must be a positive multiple of 128");
    MlpBatch bt(B, s);
    AGB_CUDA(cudaMemcpyAsync(bt.x, x, sizeof(float) * B * NIN, cudaMemcpyDefault, s));
    AGB_CUDA(cudaMemcpyAsync(bt.t, t, sizeof(float) * B * NOUT, cudaMemcpyDefault, s));
    AGB_CUDA(cudaMemcpyAsync(bt.m, m, sizeof(float) * B * NOUT, cudaMemcpyDefault, s));
    std::vector<float> hm(B * NOUT);
    AGB_CUDA(cudaMemcpyAsync(hm.data(), m, sizeof(float) * B * NOUT, cudaMemcpyDefault, s));
    AGB_CUDA(cudaStreamSynchronize(s));
    float S = 0;
    for(float v : hm) S += v;
    AGB_CUDA(cudaMemcpyAsync(bt.maskSum, &S, sizeof(float), cudaMemcpyHostToDevice, s));
    AGB_CUDA(cudaMemsetAsync(bt.loss, 0, sizeof(float), s));
    lossGrad(bt, bt.maskSum, bt.loss, grad, s);
    float loss = 0;
    AGB_CUDA(cudaMemcpyAsync(&loss, bt.loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    AGB_CUDA(cudaStreamSynchronize(s));
    checkGemmError();
    return loss;
}

std::vector<float> Mlp::train(long n, const float* x, const float* t, const float* m, int epochs, int batch,
    float lr, unsigned long long seed, cudaStream_t s)
{
    if(batch <= 0 || batch % 128) throw std::invalid_argument("mlp: the batch size must be a positive multiple of 128");
    if(n < batch) throw std::invalid_argument("mlp: fewer training samples than one batch");
    // standardisation from the data (masked for the targets), host side
    std::vector<float> hx(n * NIN), ht(n * NOUT), hm(n * NOUT);
    AGB_CUDA(cudaMemcpyAsync(hx.data(), x, sizeof(float) * n * NIN, cudaMemcpyDefault, s));
    AGB_CUDA(cudaMemcpyAsync(ht.data(), t, sizeof(float) * n * NOUT, cudaMemcpyDefault, s));
    AGB_CUDA(cudaMemcpyAsync(hm.data(), m, sizeof(float) * n * NOUT, cudaMemcpyDefault, s));
    AGB_CUDA(cudaStreamSynchronize(s));
    std::vector<float> sc(2 * NIN + 2 * NOUT);
    for(int k = 0; k < NIN; k++) {
        double s1 = 0, s2 = 0;
        for(long i = 0; i < n; i++) { s1 += hx[i * NIN + k]; s2 += double(hx[i * NIN + k]) * hx[i * NIN + k]; }
        const double mu = s1 / n, sd = std::sqrt(std::max(s2 / n - mu * mu, 1e-30));
        sc[k] = static_cast<float>(mu); sc[NIN + k] = static_cast<float>(sd);
    }
    for(int j = 0; j < NOUT; j++) {
        double s0 = 0, s1 = 0, s2 = 0;
        for(long i = 0; i < n; i++) if(hm[i * NOUT + j] > 0) { s0++; s1 += ht[i * NOUT + j]; s2 += double(ht[i * NOUT + j]) * ht[i * NOUT + j]; }
        const double mu = s0 > 0 ? s1 / s0 : 0, sd = s0 > 0 ? std::sqrt(std::max(s2 / s0 - mu * mu, 1e-30)) : 1;
        sc[2 * NIN + j] = static_cast<float>(mu); sc[2 * NIN + NOUT + j] = static_cast<float>(sd);
    }
    AGB_CUDA(cudaMemcpy(scaling.ptr, sc.data(), sizeof(float) * sc.size(), cudaMemcpyHostToDevice));
    // standardised copies of the whole set on the device
    Scratch data(sizeof(float) * n * (NIN + 2 * NOUT) + 1024, s);
    float* xs = static_cast<float*>(data.ptr);
    float* ts = xs + n * NIN;
    float* ms = ts + n * NOUT;
    AGB_CUDA(cudaMemcpyAsync(ms, m, sizeof(float) * n * NOUT, cudaMemcpyDefault, s));
    Scratch raw(sizeof(float) * n * (NIN + NOUT), s);
    float* rx = static_cast<float*>(raw.ptr);
    float* rt = rx + n * NIN;
    AGB_CUDA(cudaMemcpyAsync(rx, x, sizeof(float) * n * NIN, cudaMemcpyDefault, s));
    AGB_CUDA(cudaMemcpyAsync(rt, t, sizeof(float) * n * NOUT, cudaMemcpyDefault, s));
    standardiseKernel<<<blocks(n * NIN, 256), 256, 0, s>>>(n, NIN, rx, scaling.ptr, scaling.ptr + NIN, xs);
    standardiseKernel<<<blocks(n * NOUT, 256), 256, 0, s>>>(n, NOUT, rt, scaling.ptr + 2 * NIN, scaling.ptr + 2 * NIN + NOUT, ts);
    AGB_CUDA(cudaGetLastError());

    MlpBatch bt(batch, s);
    DevBuf<float> grad(NPARAM);
    DevBuf<int> perm(n);
    DevBuf<TrainState> state(1);
    {
        TrainState init{ 0, static_cast<int>(adamStep), 0.f, lr, 0.f, 0.f };
        AGB_CUDA(cudaMemcpyAsync(state.ptr, &init, sizeof(TrainState), cudaMemcpyHostToDevice, s));
    }
    std::mt19937_64 rng(seed);
    std::vector<int> hperm(n);
    for(long i = 0; i < n; i++) hperm[i] = static_cast<int>(i);
    std::vector<float> history;
    const long steps = n / batch;
    // one Adam step (gather, forward, backward, update, BF16 weight copies, counters) captured once
    // and replayed: it reads its batch index, mask sum, learning rate and step count from the state
    prepareGemm();
    cudaStream_t cs;
    AGB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    AGB_CUDA(cudaStreamSynchronize(s));
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    try {
        AGB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        gatherBatchKernel<<<blocks(batch, 256), 256, 0, cs>>>(batch, perm.ptr, state.ptr, xs, ts, ms, bt.x, bt.t, bt.m);
        lossGrad(bt, &state.ptr->maskSum, &state.ptr->loss, grad.ptr, cs);
        adamKernel<<<blocks(NPARAM, 256), 256, 0, cs>>>(NPARAM, params.ptr, grad.ptr, adamM.ptr, adamV.ptr, state.ptr,
            0.9f, 0.999f, 1e-8f);
        refreshWeights(cs);
        finishStepKernel<<<1, 1, 0, cs>>>(state.ptr);
        AGB_CUDA(cudaStreamEndCapture(cs, &graph));
        AGB_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        for(int e = 0; e < epochs; e++) {
            std::shuffle(hperm.begin(), hperm.end(), rng);
            AGB_CUDA(cudaMemcpyAsync(perm.ptr, hperm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, cs));
            const float lrE = lr * 0.5f * (1 + std::cos(static_cast<float>(M_PI) * e / std::max(1, epochs)));   // cosine decay
            startEpochKernel<<<1, 1, 0, cs>>>(state.ptr, lrE);
            AGB_CUDA(cudaGetLastError());
            for(long st = 0; st < steps; st++) AGB_CUDA(cudaGraphLaunch(exec, cs));
            TrainState h;
            AGB_CUDA(cudaMemcpyAsync(&h, state.ptr, sizeof(TrainState), cudaMemcpyDeviceToHost, cs));
            AGB_CUDA(cudaStreamSynchronize(cs));
            history.push_back(static_cast<float>(h.lossSum / steps));
            adamStep = h.adamStep;
        }
    } catch(...) {
        if(exec) cudaGraphExecDestroy(exec);
        if(graph) cudaGraphDestroy(graph);
        cudaStreamDestroy(cs);
        throw;
    }
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    AGB_CUDA(cudaStreamDestroy(cs));
    AGB_CUDA(cudaStreamSynchronize(s));
    checkGemmError();
    return history;
}

void Mlp::predict(long n, const float* x, float* y, cudaStream_t s) const
{
    if(n <= 0) return;
    {
        // the kernel's shared-memory limit is a per-device attribute: raise it once per device
        static std::mutex mtx;
        static std::set<int> raised;
        std::lock_guard<std::mutex> lock(mtx);
        if(!raised.count(device)) {
            AGB_CUDA(cudaFuncSetAttribute(mlpInferKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, INF_SMEM));
            raised.insert(device);
        }
    }
    int sms = 0;
    AGB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const long tiles = (n + 127) / 128;
    const int grid = static_cast<int>(std::min<long>(tiles, 2L * sms));
    mlpInferKernel<<<grid, INF_THREADS, INF_SMEM, s>>>(n, x, y, params.ptr, reinterpret_cast<const __nv_bfloat16*>(w2.ptr),
        reinterpret_cast<const __nv_bfloat16*>(w3.ptr), scaling.ptr, error.ptr);
    AGB_CUDA(cudaGetLastError());
}

void Mlp::checkError() const
{
    int h = 0;
    AGB_CUDA(cudaMemcpy(&h, error.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    if(h) {
        AGB_CUDA(cudaMemset(error.ptr, 0, sizeof(int)));      // reported once
        throw std::runtime_error("mlp: tensor-core completion barrier timed out");
    }
}

}  // namespace agb
