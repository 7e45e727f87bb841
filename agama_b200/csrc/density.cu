// Density of a Multipole potential (the reference's agama_evalDensity on a potential object,
// src/interface_c.cpp:63-66 -> Multipole::densityCyl, src/potential_multipole.cpp:1550-1559),
// batched: one point per thread.
//
// Inside the radial grid the density is the Laplacian of the interpolated potential divided by
// 4 pi (BasePotential::densityCyl, src/potential_base.cpp:51-75); outside it, the power-law
// asymptotic expansions give it in closed form (PowerLawMultipole::densityCyl,
// src/potential_multipole.cpp:1660-1687).
#include "runtime.h"
#include "multipole_eval.cuh"

namespace agb {

namespace {

constexpr int DENSITY_BLOCK = 128;
constexpr double SQRT_DBL_EPS = 1.4901161193847656e-08;          // sqrt(DBL_EPSILON)
constexpr double EPSREL_DENSITY_DER = 3.666852862501036e-11;     // DBL_EPSILON / DBL_EPSILON^(1/3)

/// value of the spherical-harmonic series sum_lm C_lm Y_lm(tau, phi) with C_lm from coef(c)
/// (math::sphHarmTransformInverse, src/math_sphharm.cpp:386-414)
template<class Coef>
__device__ double sphHarmValue(const HarmIndices& ind, const Coef& coef, double tau, double phi)
{
    double trig[2 * LMAX_MAX];
    double P[LMAX_MAX + 1];
    const bool useSine = ind.mmin() < 0;
    if(ind.mmax > 0) trigMultiAngle(phi, ind.mmax, useSine, trig);
    double result = 0;
    for(int m = ind.mmin(); m <= ind.mmax; m++) {
        const int lmin = ind.lmin(m);
        if(lmin > ind.lmax) continue;
        const int absm = m < 0 ? -m : m;
        const double t = m == 0 ? 2 * SQRT_PI :
            m > 0 ? trig[m - 1] * (2 * SQRT_PI * M_SQRT2) : trig[ind.mmax - m - 1] * (2 * SQRT_PI * M_SQRT2);
        legendreArray(ind.lmax, absm, tau, P, nullptr, nullptr);
        for(int l = lmin; l <= ind.lmax; l += ind.step)
            result += coef(HarmIndices::index(l, m)) * P[l - absm] * t;
    }
    return result;
}

/// closed-form density of a power-law expansion (PowerLawMultipole::densityCyl)
__device__ double powerLawDensity(const PowerLawView& A, double R, double z, double phi)
{
    const HarmIndices& ind = A.ind;
    const double rsq = R * R + z * z, dlogr = log(rsq / A.r0sq) * 0.5;
    const int lmax = (A.inner && rsq < A.r0sq * 1e-16) || (!A.inner && rsq > A.r0sq * 1e16) ? 0 : ind.lmax;
    auto rho = [&](int c) {
        const int l = static_cast<int>(sqrt(static_cast<double>(c)));
        const double s = ldg(A.S + c), u = ldg(A.U + c), v = A.inner ? l : -l - 1;
        const double ursm2 = s != 2 ? u * exp(dlogr * (s - 2)) : u;     // u (r/r0)^(s-2)
        if(s != v)
            return ursm2 * (s * (s + 1) - l * (l + 1)) + (v == 0 ? 6 * A.Q : 0);
        return ursm2 * (s * (s + 1) * dlogr - s * (s - 1) + 1);
    };
    if(lmax == 0)
        return 0.25 / M_PI / A.r0sq * rho(0);
    const double tau = z == 0 ? 0 : z / (sqrt(R * R + z * z) + R);
    return 0.25 / M_PI / A.r0sq * sphHarmValue(ind, rho, tau, phi);
}

/// gradient and Hessian of the interpolated potential inside the grid (the interpolator alone,
/// as the reference's impl object)
template<int KIND>
__device__ __forceinline__ void interiorDerivs(const MultipoleView& M, double R, double z, double phi,
    CylDerivs* g, CylHess* h)
{
    double Phi;
    if(M.is2d) {
        if(KIND == EVAL_AXI)       evalInterp2dFast<6, 1>(M, R, z, phi, &Phi, g, h);
        else if(KIND == EVAL_FAST) evalInterp2dFast<6, FAST_MAX_HARMONICS>(M, R, z, phi, &Phi, g, h);
        else                       evalInterp2d<6>(M, R, z, phi, &Phi, g, h);
    } else
        evalInterp1d<6>(M, R, z, phi, &Phi, g, h);
}

/// Laplacian / (4 pi) in cylindrical coordinates with the reference's treatment of the z axis
/// and of results dominated by round-off (BasePotential::densityCyl)
template<int KIND>
__device__ double laplacianDensity(const MultipoleView& M, double R, double z, double phi)
{
    CylDerivs g; CylHess h;
    interiorDerivs<KIND>(M, R, z, phi, &g, &h);
    double dRoverR = g.dR / R;
    double d2phiOverR2 = h.dphi2 / pow2(R);
    if(R <= fabs(z) * SQRT_DBL_EPS) {        // on or next to the z axis
        dRoverR = h.dR2;
        if((M.ind.sym & SYM_ZROT) == SYM_ZROT)
            d2phiOverR2 = 0;
        else {                               // d2Phi/dphi2 from a point just off the axis
            const double Roff = fabs(z) * SQRT_DBL_EPS;
            CylDerivs go; CylHess ho;
            interiorDerivs<KIND>(M, Roff, z, phi, &go, &ho);
            d2phiOverR2 = ho.dphi2 / pow2(Roff);
        }
    }
    const double result = h.dR2 + dRoverR + h.dz2 + d2phiOverR2;
    if(!(fabs(result) > EPSREL_DENSITY_DER * (fabs(h.dR2) + fabs(dRoverR) + fabs(h.dz2) + fabs(d2phiOverR2))))
        return 0;
    return result / (4 * M_PI);
}

template<int KIND>
__global__ void __launch_bounds__(DENSITY_BLOCK) densityKernel(const __grid_constant__ MultipoleView M, long n,
    const double* __restrict__ pos, double* __restrict__ rho)
{
    const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if(i >= n) return;
    const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    const double R = sqrt(x * x + y * y), phi = atan2(y, x);      // coord::toPosCyl
    const double rsq = R * R + z * z;
    double d;
    if(rsq < M.rInnerSq)      d = powerLawDensity(M.inner, R, z, phi);
    else if(rsq > M.rOuterSq) d = powerLawDensity(M.outer, R, z, phi);
    else                      d = laplacianDensity<KIND>(M, R, z, phi);
    rho[i] = d;
}

}  // namespace

void launchDensity(const MultipoleView& M, long n, const double* pos, double* rho, cudaStream_t stream)
{
    if(n <= 0) return;
    const long grid = (n + DENSITY_BLOCK - 1) / DENSITY_BLOCK;
    const int kind = evalKindOf(M);
    if(kind == EVAL_AXI)       densityKernel<EVAL_AXI><<<grid, DENSITY_BLOCK, 0, stream>>>(M, n, pos, rho);
    else if(kind == EVAL_FAST) densityKernel<EVAL_FAST><<<grid, DENSITY_BLOCK, 0, stream>>>(M, n, pos, rho);
    else                       densityKernel<EVAL_GENERAL><<<grid, DENSITY_BLOCK, 0, stream>>>(M, n, pos, rho);
    AGB_CUDA(cudaGetLastError());
}

}  // namespace agb
