// Phase 3 of the Staeckel-fudge actions: the Gauss-Legendre action integrals.  In its own
// compilation unit so that its register budget does not constrain the other phases (the
// potential evaluator is a non-inlined function compiled once per unit).
#include "runtime.h"
#include "fudge.cuh"
#include "fudge_phases.h"
#include <algorithm>
#include <map>
#include <mutex>

namespace agb {

namespace {

constexpr int INTEGRAL_BLOCK = 128;
constexpr unsigned FULL_MASK = 0xffffffffu;

/// Phase 3: every action integral (task t < n: Jr of point t; t >= n: Jz of point t - n) drained
/// from one work counter by a persistent grid.  A lane evaluates one Gauss-Legendre node of its
/// integral per step and takes the next integral as soon as its last node is summed, so that
/// integrals of different orders (10 to 40 nodes) keep every lane busy.  The nodes of one integral
/// are summed in order (computeActions, src/actions_staeckel.cpp:604-619: Jr = I_lambda / pi,
/// Jz = 2 I_nu / pi).
/// MIXED: the integrand's arithmetic after F(tau) in FP32 (fudgeMomentumNode32) and the weighted
/// terms summed in FP32 with a compensation term (Kahan), converted to FP64 at the end.
template<bool MIXED>
__global__ void __launch_bounds__(INTEGRAL_BLOCK, 5) fudgeIntegralKernel(const __grid_constant__ MultipoleView M,
    const __grid_constant__ GLRules gl, long n, const FudgeRecord* __restrict__ rec, double* __restrict__ act,
    unsigned long long* __restrict__ counter)
{
    const long total = 2 * n;
    const unsigned lane = threadIdx.x & 31;
    bool busy = false, drained = false;
    long point = 0;
    int which = 0, node = 0, numNodes = 0;
    double lo = 0, hi = 0, sum = 0;
    float sum32 = 0.f, comp32 = 0.f;
    const double* x = nullptr;
    const double* w = nullptr;
    FudgeFunction fnc;
    while(true) {
        while(true) {
            const unsigned need = __ballot_sync(FULL_MASK, !busy && !drained);
            if(!need) break;
            const int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if(static_cast<int>(lane) == leader) base = atomicAdd(counter, static_cast<unsigned long long>(__popc(need)));
            base = __shfl_sync(FULL_MASK, base, leader);
            if(!busy && !drained) {
                const long t = static_cast<long>(base) + __popc(need & ((1u << lane) - 1));
                if(t >= total) drained = true;
                else {
                    which = t >= n;
                    point = t - which * n;
                    const FudgeRecord& r = rec[point];
                    if(r.valid) {
                        loadFudgeFunction(M, r, fnc);
                        const FudgeLimits lim = fudgeLimitsFinish(r);
                        lo = which == 0 ? lim.lambda_min : 0;
                        hi = which == 0 ? lim.lambda_max : lim.nu_max;
                        int N = lim.order < 1 ? 1 : lim.order;
                        while(gl.offset[N] < 0) N++;
                        numNodes = N;
                        x = gl.nodes + gl.offset[N];
                        w = gl.weights + gl.offset[N];
                        node = 0;
                        sum = 0;
                        sum32 = comp32 = 0.f;
                        busy = true;
                    }
                }
            }
        }
        if(!__any_sync(FULL_MASK, busy)) break;
        if(busy) {
            if(MIXED) {
                const float term = static_cast<float>(ldg(w + node)) * fudgeMomentumNode32(fnc, lo, hi, ldg(x + node));
                const float y = term - comp32, t = sum32 + y;
                comp32 = (t - sum32) - y;
                sum32 = t;
            } else
                sum += ldg(w + node) * fudgeMomentumNode(fnc, lo, hi, ldg(x + node));
            if(++node == numNodes) {
                busy = false;
                if(MIXED) sum = static_cast<double>(sum32) - static_cast<double>(comp32);
                act[3 * point + which] = which == 0 ? sum / M_PI : sum / M_PI * 2;
            }
        }
    }
}

/// resident blocks of the integral kernel on the current device (cached per device and variant)
template<bool MIXED>
int integralGridSize()
{
    static std::mutex mutex;
    static std::map<int, int> cache;
    int dev;
    AGB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mutex);
    auto it = cache.find(dev);
    if(it != cache.end()) return it->second;
    int sms = 0, perSM = 0;
    AGB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    AGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fudgeIntegralKernel<MIXED>, INTEGRAL_BLOCK, 0));
    const int grid = std::max(1, sms * std::max(1, perSM));
    cache[dev] = grid;
    return grid;
}

}  // namespace

void launchFudgeIntegrals(const MultipoleView& M, const GLRules& gl, long n, const FudgeRecord* rec, double* act,
    unsigned long long* counter, bool mixed, cudaStream_t stream)
{
    if(n <= 0) return;
    AGB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), stream));
    const long tasks = (2 * n + INTEGRAL_BLOCK - 1) / INTEGRAL_BLOCK;
    if(mixed) {
        const long grid = std::min<long>(integralGridSize<true>(), tasks);
        fudgeIntegralKernel<true><<<grid, INTEGRAL_BLOCK, 0, stream>>>(M, gl, n, rec, act, counter);
    } else {
        const long grid = std::min<long>(integralGridSize<false>(), tasks);
        fudgeIntegralKernel<false><<<grid, INTEGRAL_BLOCK, 0, stream>>>(M, gl, n, rec, act, counter);
    }
    AGB_CUDA(cudaGetLastError());
}

}  // namespace agb
