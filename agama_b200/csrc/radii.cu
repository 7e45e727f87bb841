// Radii of circular, radial and planar orbits of a potential (the reference's potential_utils
// routines behind agama_R_circ, agama_R_from_Lz, agama_R_max and agama_findPlanarOrbitExtent,
// src/interface_c.cpp:92-111 -> src/potential_utils.cpp:617-729), batched: one query per thread.
//
// Every query works in the equatorial plane of the potential averaged over the azimuth
// (Axisymmetrized<BasePotential>, src/potential_base.h:449-472): an axisymmetric potential is
// evaluated directly at phi = 0; any other is averaged over 2*8+1 equally spaced azimuths
// (azimuthalAverage, src/potential_base.cpp:256-283), with the same points, weights and
// summation order as the reference.
#include "runtime.h"
#include "shell.cuh"

namespace agb {

namespace {

constexpr int RADII_BLOCK = 128;

/// the potential at (R, z = 0, phi = 0) with its R-derivatives, for an axisymmetric Multipole
/// (KIND: the spline evaluator that matches the potential)
template<int KIND>
struct DirectRadial {
    const MultipoleView* M;
    __device__ void operator()(double R, double* val, double* der, double* der2) const {
        double Phi;
        CylDerivs g; CylHess h;
        if(der2)     evalMultipoleCylCall<6, KIND>(*M, R, 0, 0, &Phi, &g, &h);
        else if(der) evalMultipoleCylCall<3, KIND>(*M, R, 0, 0, &Phi, &g, &h);
        else         evalMultipoleCylCall<1, KIND>(*M, R, 0, 0, &Phi, &g, &h);
        if(val) *val = Phi;
        if(der) *der = g.dR;
        if(der2) *der2 = h.dR2;
    }
};

/// Axisymmetrized<BasePotential>::evalCyl at z = 0 for a potential without z-rotation symmetry
/// (src/potential_base.cpp:529-590): nothing to average at R = 0 or R = inf; otherwise the
/// mean over phi_i = pi / (nphi + 1/2) * i, i = 0..2 nphi (nphi = 8), where with y-reflection
/// symmetry the points i = 1..nphi carry weight 2 and stand for their mirror images
struct AveragedRadial {
    const MultipoleView* M;
    int ysym;
    __device__ void operator()(double R, double* val, double* der, double* der2) const {
        double Phi;
        CylDerivs g; CylHess h;
        if(R == 0 || R == INFINITY) {
            evalMultipoleCylCall<6, EVAL_GENERAL>(*M, R, 0, 0, &Phi, &g, &h);
            if(val) *val = Phi;
            if(der) *der = g.dR;
            if(der2) *der2 = h.dR2;
            return;
        }
        const int nphi = 8, npoints = ysym ? nphi + 1 : 2 * nphi + 1;
        double sv = 0, sd = 0, sh = 0;
        for(int i = 0; i < npoints; i++) {
            const double phi = M_PI / (nphi + 0.5) * i;
            if(der2)     evalMultipoleCylCall<6, EVAL_GENERAL>(*M, R, 0, phi, &Phi, &g, &h);
            else if(der) evalMultipoleCylCall<3, EVAL_GENERAL>(*M, R, 0, phi, &Phi, &g, &h);
            else         evalMultipoleCylCall<1, EVAL_GENERAL>(*M, R, 0, phi, &Phi, &g, &h);
            const double w = ysym && i > 0 ? 2 : 1;
            sv += Phi * w;
            if(der) sd += g.dR * w;
            if(der2) sh += h.dR2 * w;
        }
        const double norm = 1. / (2 * nphi + 1);
        if(val) *val = sv * norm;
        if(der) *der = sd * norm;
        if(der2) *der2 = sh * norm;
    }
};

template<class EV>
__device__ __forceinline__ void radiusQuery(const EV& ev, int query, double a, double b, double* r1, double* r2)
{
    switch(query) {
        case RADIUS_CIRC_E: *r1 = radiusCirc(ev, a); break;
        case RADIUS_CIRC_L: *r1 = radiusFromLz(ev, a); break;
        case RADIUS_MAX:    *r1 = radiusMax(ev, a); break;
        default: {
            double R1, R2;
            planarOrbitExtent(ev, a, b, R1, R2);
            *r1 = R1; *r2 = R2;
        }
    }
}

/// one query per thread: a = E (or L for RADIUS_CIRC_L), b = L for RADIUS_PERIAPO;
/// out1 = the radius (the pericentre), out2 = the apocentre
template<int KIND, bool AVG>
__global__ void __launch_bounds__(RADII_BLOCK) radiiKernel(const __grid_constant__ MultipoleView M, int ysym,
    int query, long n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out1,
    double* __restrict__ out2)
{
    const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if(i >= n) return;
    double r1 = NAN, r2 = NAN;
    const double bi = query == RADIUS_PERIAPO ? b[i] : 0;
    if(AVG) radiusQuery(AveragedRadial{ &M, ysym }, query, a[i], bi, &r1, &r2);
    else    radiusQuery(DirectRadial<KIND>{ &M }, query, a[i], bi, &r1, &r2);
    out1[i] = r1;
    if(query == RADIUS_PERIAPO) out2[i] = r2;
}

}  // namespace

void launchRadii(const MultipoleView& M, int query, long n, const double* a, const double* b, double* out1,
    double* out2, cudaStream_t stream)
{
    if(n <= 0) return;
    if(query < RADIUS_CIRC_E || query > RADIUS_PERIAPO)
        throw std::invalid_argument("radii: unknown query " + std::to_string(query));
    const long grid = (n + RADII_BLOCK - 1) / RADII_BLOCK;
    const bool zrot = (M.ind.sym & SYM_ZROT) == SYM_ZROT;
    const int ysym = (M.ind.sym & SYM_YREFL) == SYM_YREFL;
    if(!zrot)
        radiiKernel<EVAL_GENERAL, true><<<grid, RADII_BLOCK, 0, stream>>>(M, ysym, query, n, a, b, out1, out2);
    else if(evalKindOf(M) == EVAL_AXI)
        radiiKernel<EVAL_AXI, false><<<grid, RADII_BLOCK, 0, stream>>>(M, ysym, query, n, a, b, out1, out2);
    else
        radiiKernel<EVAL_GENERAL, false><<<grid, RADII_BLOCK, 0, stream>>>(M, ysym, query, n, a, b, out1, out2);
    AGB_CUDA(cudaGetLastError());
}

}  // namespace agb
