// Multipole potential on the device: table upload and the batched evaluation kernel.
#include "runtime.h"
#include "multipole_eval.cuh"

namespace agb {

namespace {
thread_local std::string g_error;

/// One point per thread; 256 threads per block.  NQ = 1 (potential), 3 (+gradient), 6 (+Hessian);
/// KIND = spline evaluator matching the potential (EvalKind).
template<int NQ, int KIND>
__global__ void __launch_bounds__(128) evalPotentialKernel(const MultipoleView M, long n,
    const double* __restrict__ pos, double* __restrict__ phi, double* __restrict__ grad,
    double* __restrict__ hess)
{
    const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if(i >= n) return;
    const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    double p, g[3], h[6];
    evalMultipoleCar<NQ, KIND>(M, x, y, z, &p, g, h);
    if(phi) phi[i] = p;
    if(NQ >= 3 && grad) { grad[3 * i] = g[0]; grad[3 * i + 1] = g[1]; grad[3 * i + 2] = g[2]; }
    if(NQ == 6 && hess)
        for(int k = 0; k < 6; k++) hess[6 * i + k] = h[k];
}

/// the same at n cylindrical points (R, z, phi), derivatives in cylindrical coordinates
/// (dR, dz, dphi; dR2, dz2, dphi2, dRdz, dzdphi, dRdphi) straight from the evaluator, as the
/// reference's BasePotentialCyl::evalCyl returns them (no round trip through Cartesian
/// derivatives, which loses the phi derivatives to cancellation at large R)
template<int NQ, int KIND>
__global__ void __launch_bounds__(128) evalPotentialCylKernel(const MultipoleView M, long n,
    const double* __restrict__ pos, double* __restrict__ phi, double* __restrict__ grad,
    double* __restrict__ hess)
{
    const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if(i >= n) return;
    double p;
    CylDerivs g; CylHess h;
    evalMultipoleCyl<NQ, KIND>(M, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], &p, &g, &h);
    if(phi) phi[i] = p;
    if(NQ >= 3 && grad) { grad[3 * i] = g.dR; grad[3 * i + 1] = g.dz; grad[3 * i + 2] = g.dphi; }
    if(NQ == 6 && hess) {
        hess[6 * i] = h.dR2; hess[6 * i + 1] = h.dz2; hess[6 * i + 2] = h.dphi2;
        hess[6 * i + 3] = h.dRdz; hess[6 * i + 4] = h.dzdphi; hess[6 * i + 5] = h.dRdphi;
    }
}
}  // namespace

void setError(const std::string& msg) { g_error = msg; }
const char* lastError() { return g_error.c_str(); }

void requireDevice()
{
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if(e != cudaSuccess || count == 0)
        throw std::runtime_error("no CUDA device available: the B200 engine has no CPU fallback");
}

void launchEvalPotential(const MultipoleView& M, long n, const double* pos, double* phi,
    double* grad, double* hess, cudaStream_t stream, bool cylindrical)
{
    if(n <= 0) return;
    // 128 threads (up to 168 registers, no spills for the multi-harmonic kind): 16 % faster than
    // blocks of 256 at 128 registers with spills (config 1 forces 0.055 against 0.065 ms)
    const int block = 128;
    const long grid = (n + block - 1) / block;
    const int nq = hess ? 6 : grad ? 3 : 1, kind = evalKindOf(M);
#define AGB_LAUNCH(NQ_, K_) \
    (cylindrical ? evalPotentialCylKernel<NQ_, K_><<<grid, block, 0, stream>>>(M, n, pos, phi, grad, hess) \
                 : evalPotentialKernel<NQ_, K_><<<grid, block, 0, stream>>>(M, n, pos, phi, grad, hess))
    if(kind == EVAL_AXI)       { if(nq == 6) AGB_LAUNCH(6, EVAL_AXI);     else if(nq == 3) AGB_LAUNCH(3, EVAL_AXI);     else AGB_LAUNCH(1, EVAL_AXI); }
    else if(kind == EVAL_FAST) { if(nq == 6) AGB_LAUNCH(6, EVAL_FAST);    else if(nq == 3) AGB_LAUNCH(3, EVAL_FAST);    else AGB_LAUNCH(1, EVAL_FAST); }
    else                       { if(nq == 6) AGB_LAUNCH(6, EVAL_GENERAL); else if(nq == 3) AGB_LAUNCH(3, EVAL_GENERAL); else AGB_LAUNCH(1, EVAL_GENERAL); }
#undef AGB_LAUNCH
    AGB_CUDA(cudaGetLastError());
}

DevicePotential* createDevicePotential(const std::vector<double>& radii,
    const std::vector<std::vector<double>>& Phi, const std::vector<std::vector<double>>& dPhi)
{
    requireDevice();
    DevicePotential* P = new DevicePotential;
    try {
        AGB_CUDA(cudaGetDevice(&P->device));
        P->host = buildMultipole(radii, Phi, dPhi);
        const MultipoleHost& H = P->host;
        P->lnr.upload(H.lnr);
        P->tau.upload(H.tau);
        // reciprocal interval widths (IEEE division on the host and on the device give the same
        // correctly rounded value, so the spline segments built from them are bit-identical)
        auto invWidths = [](const std::vector<double>& g) {
            std::vector<double> w(g.size() > 1 ? g.size() - 1 : 1, 0.0);
            for(size_t k = 0; k + 1 < g.size(); k++) w[k] = 1 / (g[k + 1] - g[k]);
            return w;
        };
        P->lnrInvH.upload(invWidths(H.lnr));
        P->tauInvH.upload(invWidths(H.tau));
        P->spl2d.upload(H.spl2d);
        P->spl2d32.upload(std::vector<float>(H.spl2d.begin(), H.spl2d.end()));
        P->spl1d.upload(H.spl1d);
        P->innerS.upload(H.inner.S); P->innerU.upload(H.inner.U); P->innerW.upload(H.inner.W);
        P->outerS.upload(H.outer.S); P->outerU.upload(H.outer.U); P->outerW.upload(H.outer.W);
        MultipoleView& V = P->view;
        V.ind = H.ind;
        V.is2d = H.is2d;
        // switching radii (reference src/potential_multipole.cpp:1538-1548, GRID_SAFETY_FACTOR = eps^(1/3))
        const double gsf = 6.0554544523933395e-06;
        V.rInnerSq = pow2(H.radii.front() * (1 + gsf));
        V.rOuterSq = pow2(H.radii.back() * (1 - gsf));
        V.nr = static_cast<int>(H.lnr.size());
        V.lnr = P->lnr.ptr;
        V.nt = static_cast<int>(H.tau.size());
        V.tau = P->tau.ptr;
        V.lnrInvH = P->lnrInvH.ptr;
        V.tauInvH = P->tauInvH.ptr;
        auto guessScale = [](const std::vector<double>& g) {
            return g.size() > 1 ? static_cast<double>(g.size() - 1) / (g.back() - g.front()) : 0.0;
        };
        V.lnrScale = guessScale(H.lnr);
        V.tauScale = guessScale(H.tau);
        for(int i = 0; i < 2 * LMAX_MAX + 1; i++) V.splSlot[i] = H.splSlot[i];
        V.spl2d = P->spl2d.ptr;
        V.spl2d32 = P->spl2d32.ptr;
        V.spl1d = P->spl1d.ptr;
        V.logScaling = H.logScaling;
        V.invPhi0 = H.invPhi0;
        V.inner.ind = H.inner.ind; V.inner.r0sq = H.inner.r0sq; V.inner.inner = 1; V.inner.Q = H.inner.Q;
        V.inner.S = P->innerS.ptr; V.inner.U = P->innerU.ptr; V.inner.W = P->innerW.ptr;
        V.outer.ind = H.outer.ind; V.outer.r0sq = H.outer.r0sq; V.outer.inner = 0; V.outer.Q = H.outer.Q;
        V.outer.S = P->outerS.ptr; V.outer.U = P->outerU.ptr; V.outer.W = P->outerW.ptr;
        P->axisymmetric = (H.ind.sym & SYM_AXISYMMETRIC) == SYM_AXISYMMETRIC;
        // register-resident evaluator: m = 0 first, then ascending m
        V.nFast = 0;
        if(H.is2d && H.splSlot[H.ind.mmax] >= 0) {
            std::vector<int> ms(1, 0);
            for(int m = -H.ind.mmax; m <= H.ind.mmax; m++)
                if(m != 0 && H.splSlot[m + H.ind.mmax] >= 0) ms.push_back(m);
            if(static_cast<int>(ms.size()) <= FAST_MAX_HARMONICS) {
                V.nFast = static_cast<int>(ms.size());
                for(int s = 0; s < V.nFast; s++) { V.fastM[s] = ms[s]; V.fastSlot[s] = H.splSlot[ms[s] + H.ind.mmax]; }
            }
        }
        for(int s = V.nFast; s < FAST_MAX_HARMONICS; s++) { V.fastM[s] = 0; V.fastSlot[s] = 0; }
    } catch(...) {
        delete P;
        throw;
    }
    return P;
}

}  // namespace agb
