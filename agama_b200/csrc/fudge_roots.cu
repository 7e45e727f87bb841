// Phase 2 of the Staeckel-fudge actions: the root searches of the integration limits.  In its
// own compilation unit so that its register budget does not constrain the other phases (the
// potential evaluator is a non-inlined function compiled once per unit).
#include "runtime.h"
#include "fudge.cuh"
#include "fudge_phases.h"

namespace agb {

namespace {

constexpr int ROOT_BLOCK = 128;

/// Phase 2, one root search of kind KIND (ROOT_NU_MAX, ROOT_LAMBDA_MIN or ROOT_LAMBDA_MAX) per
/// thread; points that need no search of this kind return at once.
template<int KIND>
__global__ void __launch_bounds__(ROOT_BLOCK, 4) fudgeRootKernel(const __grid_constant__ MultipoleView M, long n,
    FudgeRecord* __restrict__ rec, int* __restrict__ iters)
{
    const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if(i >= n) return;
    FudgeRecord& r = rec[i];
    if(!(r.roots & KIND)) return;
    FudgeFunction fnc;
    loadFudgeFunction(M, r, fnc);
    int it = 0;
    const double x = fudgeLimitRoot(fnc, r, KIND, &it);
    if(KIND == ROOT_NU_MAX) r.nuMax = x;
    else if(KIND == ROOT_LAMBDA_MIN) r.lambdaMin = x;
    else r.lambdaMax = x;
    if(iters) atomicAdd(iters + i, it);
}

}  // namespace

void launchFudgeRoots(const MultipoleView& M, long n, FudgeRecord* rec, int* iters, cudaStream_t stream)
{
    if(n <= 0) return;
    const long grid = (n + ROOT_BLOCK - 1) / ROOT_BLOCK;
    fudgeRootKernel<ROOT_NU_MAX><<<grid, ROOT_BLOCK, 0, stream>>>(M, n, rec, iters);
    fudgeRootKernel<ROOT_LAMBDA_MIN><<<grid, ROOT_BLOCK, 0, stream>>>(M, n, rec, iters);
    fudgeRootKernel<ROOT_LAMBDA_MAX><<<grid, ROOT_BLOCK, 0, stream>>>(M, n, rec, iters);
    AGB_CUDA(cudaGetLastError());
}

}  // namespace agb
