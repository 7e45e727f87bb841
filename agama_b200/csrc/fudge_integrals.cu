// Phase 3 of the Staeckel-fudge actions: the Gauss-Legendre action integrals.  In its own
// compilation unit so that its register budget does not constrain the other phases (the
// potential evaluator is a non-inlined function compiled once per unit).
#include "runtime.h"
#include "fudge.cuh"
#include "fudge_phases.h"

namespace agb {

namespace {

constexpr int INTEGRAL_BLOCK = 128;

/// Phase 3, one action integral per thread: a block covers INTEGRAL_BLOCK/2 points, its first
/// half of warps computes their Jr and the second half their Jz, so that every warp runs one
/// branch of the integrand (lambda or nu) in the same Gauss-Legendre loop of potential evaluations.
__global__ void __launch_bounds__(INTEGRAL_BLOCK, 4) fudgeIntegralKernel(const __grid_constant__ MultipoleView M,
    const __grid_constant__ GLRules gl, long n, const FudgeRecord* __restrict__ rec, double* __restrict__ act)
{
    constexpr int HALF = INTEGRAL_BLOCK / 2;
    static_assert(HALF % 32 == 0, "each warp computes one kind of integral");
    const long i = blockIdx.x * static_cast<long>(HALF) + threadIdx.x % HALF;
    const int which = threadIdx.x / HALF;
    if(i >= n) return;
    const FudgeRecord r = rec[i];
    if(!r.valid) return;
    act[3 * i + which] = fudgeIntegral(M, gl, r, which);
}

}  // namespace

void launchFudgeIntegrals(const MultipoleView& M, const GLRules& gl, long n, const FudgeRecord* rec, double* act,
    cudaStream_t stream)
{
    if(n <= 0) return;
    fudgeIntegralKernel<<<(n + INTEGRAL_BLOCK / 2 - 1) / (INTEGRAL_BLOCK / 2), INTEGRAL_BLOCK, 0, stream>>>(M, gl, n, rec, act);
    AGB_CUDA(cudaGetLastError());
}

}  // namespace agb
