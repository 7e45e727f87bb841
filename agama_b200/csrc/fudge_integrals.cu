// Phase 3 of the Staeckel-fudge actions: the Gauss-Legendre action integrals.  In its own
// compilation unit so that its register budget does not constrain the other phases (the
// potential evaluator is a non-inlined function compiled once per unit).
#include "runtime.h"
#include "fudge.cuh"
#include "fudge_phases.h"

namespace agb {

namespace {

constexpr int INTEGRAL_BLOCK = 128;

/// Phase 3, one action integral per thread (threads 2i and 2i+1: Jr and Jz of point i), all
/// threads running the same Gauss-Legendre loop of potential evaluations.
__global__ void __launch_bounds__(INTEGRAL_BLOCK, 4) fudgeIntegralKernel(const __grid_constant__ MultipoleView M,
    const __grid_constant__ GLRules gl, long n, const FudgeRecord* __restrict__ rec, double* __restrict__ act)
{
    const long t = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if(t >= 2 * n) return;
    const long i = t >> 1;
    const int which = static_cast<int>(t & 1);
    const FudgeRecord r = rec[i];
    if(!r.valid) return;
    act[3 * i + which] = fudgeIntegral(M, gl, r, which);
}

}  // namespace

void launchFudgeIntegrals(const MultipoleView& M, const GLRules& gl, long n, const FudgeRecord* rec, double* act,
    cudaStream_t stream)
{
    if(n <= 0) return;
    fudgeIntegralKernel<<<(2 * n + INTEGRAL_BLOCK - 1) / INTEGRAL_BLOCK, INTEGRAL_BLOCK, 0, stream>>>(M, gl, n, rec, act);
    AGB_CUDA(cudaGetLastError());
}

}  // namespace agb
