// Phase 2 of the Staeckel-fudge actions: the root searches of the integration limits.  In its
// own compilation unit so that its register budget does not constrain the other phases (the
// potential evaluator is a non-inlined function compiled once per unit).
#include "runtime.h"
#include "fudge.cuh"
#include "fudge_phases.h"
#include <algorithm>
#include <map>
#include <mutex>

namespace agb {

namespace {

constexpr int ROOT_BLOCK = 128;
constexpr unsigned FULL_MASK = 0xffffffffu;

/// Phase 2: every root search of the integration limits (task t = kind * n + i for the kinds
/// nu_max, lambda_min, lambda_max of point i) drained from one work counter by a persistent grid.
/// Each lane runs one search as a RootSearch state machine and takes the next task as soon as
/// its search ends, so that the lanes of a warp meet at one potential evaluation per step instead
/// of waiting for the warp's longest search.
__global__ void __launch_bounds__(ROOT_BLOCK, 4) fudgeRootKernel(const __grid_constant__ MultipoleView M, long n,
    FudgeRecord* __restrict__ rec, int* __restrict__ iters, unsigned long long* __restrict__ counter)
{
    const long total = 3 * n;
    const unsigned lane = threadIdx.x & 31;
    bool busy = false, drained = false;
    long point = 0;
    int kind = 0;
    double x = 0, u0 = 0;
    FudgeFunction fnc;
    RootSearch s;
    while(true) {
        // give every idle lane of the warp a new search (one atomic per warp and round)
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
                    const int k = static_cast<int>(t / n);
                    const long i = t - k * n;
                    const FudgeRecord& r = rec[i];
                    if(r.roots & (1 << k)) {
                        point = i;
                        kind = 1 << k;
                        loadFudgeFunction(M, r, fnc);
                        u0 = r.lambdaPos;
                        x = kind == ROOT_NU_MAX ? s.start(fabs(r.nu), r.nuUpper, FUDGE_ACCURACY_RANGE) :
                            kind == ROOT_LAMBDA_MIN ? s.start(r.lambdaLower, r.lambdaPos, FUDGE_ACCURACY_RANGE) :
                            s.start(0, 1, FUDGE_ACCURACY_RANGE);
                        busy = true;
                    }
                }
            }
        }
        if(!__any_sync(FULL_MASK, busy)) break;
        if(busy) {
            double fx, dx;
            limitRootEval(fnc, kind, u0, x, &fx, &dx);
            if(s.feed(fx, dx, &x)) {
                busy = false;
                FudgeRecord& r = rec[point];
                if(kind == ROOT_NU_MAX) r.nuMax = isFinite(s.result) ? s.result : fabs(fnc.nu);
                else if(kind == ROOT_LAMBDA_MIN) r.lambdaMin = s.result;
                else r.lambdaMax = unscaleSemiInf(u0, s.result, nullptr);
                if(iters) atomicAdd(iters + point, s.iter);
            }
        }
    }
}

/// resident blocks of the root kernel on the current device (cached per device)
int rootGridSize()
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
    AGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fudgeRootKernel, ROOT_BLOCK, 0));
    const int grid = std::max(1, sms * std::max(1, perSM));
    cache[dev] = grid;
    return grid;
}

}  // namespace

void launchFudgeRoots(const MultipoleView& M, long n, FudgeRecord* rec, int* iters, unsigned long long* counter,
    cudaStream_t stream)
{
    if(n <= 0) return;
    AGB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), stream));
    const long grid = std::min<long>(rootGridSize(), (3 * n + ROOT_BLOCK - 1) / ROOT_BLOCK);
    fudgeRootKernel<<<grid, ROOT_BLOCK, 0, stream>>>(M, n, rec, iters, counter);
    AGB_CUDA(cudaGetLastError());
}

}  // namespace agb
