// Phase 3 of the Staeckel-fudge computation when angles or frequencies are requested: actions,
// frequencies and angles of each prepared point, one point per thread.
#include "runtime.h"
#include "fudge.cuh"
#include "fudge_phases.h"

namespace agb {

namespace {

constexpr int ANGLE_BLOCK = 128;

__global__ void __launch_bounds__(ANGLE_BLOCK, 4) fudgeAngleKernel(const __grid_constant__ MultipoleView M,
    const __grid_constant__ GLRules gl, long n, const FudgeRecord* __restrict__ rec, double* __restrict__ act,
    double* __restrict__ ang, double* __restrict__ freq)
{
    const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if(i >= n) return;
    const FudgeRecord r = rec[i];
    if(!r.valid) {          // no actions (set by phase 1): angles and frequencies are NaN too
        for(int k = 0; k < 3; k++) {
            if(ang) ang[3 * i + k] = NAN;
            if(freq) freq[3 * i + k] = NAN;
        }
        return;
    }
    double a[2];
    fudgeAnglesFrequencies(M, gl, r, a, ang ? ang + 3 * i : nullptr, freq ? freq + 3 * i : nullptr);
    act[3 * i] = a[0];
    act[3 * i + 1] = a[1];
}

}  // namespace

void launchFudgeAngles(const MultipoleView& M, const GLRules& gl, long n, const FudgeRecord* rec, double* act,
    double* ang, double* freq, cudaStream_t stream)
{
    if(n <= 0) return;
    fudgeAngleKernel<<<(n + ANGLE_BLOCK - 1) / ANGLE_BLOCK, ANGLE_BLOCK, 0, stream>>>(M, gl, n, rec, act, ang, freq);
    AGB_CUDA(cudaGetLastError());
}

}  // namespace agb
