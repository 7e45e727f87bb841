// Construction of the Staeckel-fudge action finder's tables for a device-resident potential:
// the L_circ(E) interpolator (host C++ on device-evaluated potential values) and the
// focal-distance table Delta(E, Lz/Lcirc) from shell orbits (device kernel, one node per thread).
//
// Reference: potential::createInterpolationGrid / math::createInterpolationGrid
// (src/potential_utils.cpp:738-753, src/math_spline.cpp:4309-4390), potential::Interpolator
// constructor (src/potential_utils.cpp:757-870), ActionFinderAxisymFudge constructor and
// createGridFocalDistance (src/actions_staeckel.cpp:700-795).
#include "runtime.h"
#include "shell.cuh"
#include <algorithm>

namespace agb {

namespace {

constexpr double MIN_REL_DIFFERENCE = 3.666852862501036e-11;   // potential_utils.cpp:46
constexpr double ACCURACY_INTERP = 1e-6;                        // potential_utils.cpp:34
constexpr double ACCURACY_INTERP2 = 1e-4;                       // actions_staeckel.cpp:41
constexpr int SIZE_L = 25;                                      // actions_staeckel.cpp:756
constexpr double ROUNDOFF_THRESHOLD = 3.666852862501036e-11;

/// Phi, dPhi/dR, d2Phi/dR2, d2Phi/dz2 at (R_i, 0, 0)
__global__ void equatorialKernel(const __grid_constant__ MultipoleView M, int n, const double* R, double* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    double Phi;
    CylDerivs g; CylHess h;
    evalMultipoleCylCall<6, EVAL_AXI>(M, R[i], 0, 0, &Phi, &g, &h);
    out[4 * i] = Phi; out[4 * i + 1] = g.dR; out[4 * i + 2] = h.dR2; out[4 * i + 3] = h.dz2;
}

/// focal distance at each (E_i, Lz/Lcirc = L_j) node from its shell orbit
__global__ void shellGridKernel(const __grid_constant__ MultipoleView M, int nE, int nL, const double* gridE,
    const double* gridL, double* delta, double* rshell)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if(k >= nE * nL) return;
    const int iE = k / nL, iL = k % nL;
    const double E = gridE[iE];
    const double Rc = shellRcirc(M, E);
    const double vc = shellVcirc(M, Rc);
    const double Lz = Rc * vc * gridL[iL];
    double Rsh;
    delta[k] = shellFocalDistance(M, E, Lz, &Rsh);
    rshell[k] = Rsh / Rc;
}

/// host-side evaluation of the equatorial potential at a list of radii
struct Equatorial {
    const DevicePotential& P;
    DevBuf<double> dR, dOut;
    std::vector<double> eval(const std::vector<double>& R) {
        const int n = static_cast<int>(R.size());
        std::vector<double> out(4 * n);
        if(n == 0) return out;
        dR.upload(R);
        dOut.alloc(4 * n);
        equatorialKernel<<<(n + 127) / 128, 128>>>(P.view, n, dR.ptr, dOut.ptr);
        AGB_CUDA(cudaGetLastError());
        AGB_CUDA(cudaMemcpy(out.data(), dOut.ptr, 4 * n * sizeof(double), cudaMemcpyDeviceToHost));
        return out;
    }
    double value(double R) { return eval(std::vector<double>(1, R))[0]; }
};

/// second derivative of the scaled potential in ln r (ScalePhi, potential_utils.cpp:447-472)
double scalePhiDer2(Equatorial& Q, double invPhi0, double logr)
{
    const double r = exp(logr);
    const std::vector<double> v = Q.eval(std::vector<double>(1, r));
    const double Phi = v[0], dR = v[1], dR2 = v[2], dz2 = v[3];
    const double expE = invPhi0 - 1 / Phi;
    if(invPhi0 != 0 && expE < -invPhi0 * MIN_REL_DIFFERENCE)
        return 0;
    return pow2(r / Phi) / expE * (dR * (1 / r - dR / Phi * (2 + 1 / Phi / expE)) + dR2) +
        2 * r * r / Phi * (dR2 + dz2 - pow2(dR) / Phi);
}

/// grid in ln r whose spacing follows the variation of the scaled potential
/// (math::createInterpolationGrid on ScalePhi, then the inner-node trimming of
/// potential::createInterpolationGrid)
std::vector<double> interpolationGrid(Equatorial& Q, double invPhi0, double Phi0, double eps)
{
    const double xmax = 100.;
    const double XINIT[16] = { -75, -50, -32, -22, -15, -10, -6, -2, 2, 6, 10, 15, 22, 32, 50, 75 };
    double xinit = 0., d2f0 = 0., xlow = xmax, xupp = -xmax;
    for(int k = 0; k < 16; k++) {
        const double d2 = scalePhiDer2(Q, invPhi0, XINIT[k]);
        if(isFinite(d2)) {
            if(fabs(d2) > eps) { xlow = fmin(xlow, XINIT[k]); xupp = fmax(xupp, XINIT[k]); }
            if(fabs(d2) > fabs(d2f0)) { xinit = XINIT[k]; d2f0 = d2; }
        }
    }
    const double eps4 = sqrt(sqrt(eps * (384. / 5)));
    double d2fm = scalePhiDer2(Q, invPhi0, xinit - eps4);
    double d2fp = scalePhiDer2(Q, invPhi0, xinit + eps4);
    const double d3f0 = (d2f0 - d2fm) / eps4;
    double d3fp = (d2fp - d2f0) / eps4;
    float dx = -eps4;      // single precision on purpose: coarse-grains the step like the reference
    double x = xinit;
    d2fp = d2f0;
    std::vector<double> result(1, xinit);
    int stage = 0;
    while(stage < 2) {
        const double d2f = scalePhiDer2(Q, invPhi0, x + dx);
        const double d3f = (d2f - d2fp) / dx;
        const double dif = fabs((d3f - d3fp) / dx) + 0.1 * (fabs(d3fp) + fabs(d3f));
        const double sgn = (stage * 2 - 1);
        const double dxn = eps4 / fmax(fmin(sqrt(sqrt(dif)), 2.0), 0.01) * sgn;
        if(fabs(dxn / dx) <= 0.5) {
            dx = dxn;
            continue;
        }
        x += dx;
        dx = dxn;
        result.push_back(x);
        if((fabs(d2f) < eps && fabs(d2fp) < eps && ((stage == 0 && x < xlow) || (stage == 1 && x > xupp)))
            || fabs(x) > xmax || !isFinite(d2f + dx)) {
            if(stage == 0) {
                std::reverse(result.begin(), result.end());
                x = xinit;
                dx = eps4;
                d2fp = d2f0;
                d3fp = d3f0;
            }
            ++stage;
        } else {
            d2fp = d2f;
            d3fp = d3f;
        }
    }
    for(double& g : result) g = exp(g);
    while(result.size() > 2 && Q.value(result[0]) < Phi0 * (1 - MIN_REL_DIFFERENCE))
        result.erase(result.begin());
    return result;
}

void pushSpline(std::vector<double>& out, const std::vector<double>& x, const std::vector<double>& f,
    const std::vector<double>& d)
{
    const std::vector<double> d2 = quinticSecondDerivs(x, f, d);
    out.clear();
    out.insert(out.end(), x.begin(), x.end());
    out.insert(out.end(), f.begin(), f.end());
    out.insert(out.end(), d.begin(), d.end());
    out.insert(out.end(), d2.begin(), d2.end());
}

}  // namespace

FinderTablesHost buildFinderTables(const DevicePotential& P)
{
    if(!P.axisymmetric)
        throw std::invalid_argument("Fudge approximation only works for axisymmetric potentials");
    AGB_CUDA(cudaSetDevice(P.device));
    Equatorial Q{ P };
    FinderTablesHost T;
    const double Phi0 = Q.value(0);
    const double invPhi0 = 1. / Phi0;
    if(invPhi0 > 0 || !isFinite(invPhi0))
        throw std::runtime_error("ActionFinder: potential must be negative at r=0");
    T.invPhi0 = invPhi0;
    T.interpInvPhi0 = invPhi0;

    // ---- potential::Interpolator (L_circ(E) and the splines it needs)
    {
        const std::vector<double> gridR = interpolationGrid(Q, invPhi0, Phi0, ACCURACY_INTERP);
        const size_t n = gridR.size();
        const std::vector<double> v = Q.eval(gridR);
        std::vector<double> logR(n), sPhi(n), sE(n), logL(n), dRdL(n), dLdE(n), dPhi(n);
        for(size_t i = 0; i < n; i++) {
            const double R = gridR[i], Phi = v[4 * i], gR = v[4 * i + 1], hRR = v[4 * i + 2];
            logR[i] = log(R);
            const double kappa2 = hRR + 3 * gR / R, Omega = sqrt(gR / R);
            const double Ecirc = Phi + 0.5 * R * gR, Lcirc = Omega * R * R;
            const double expP = invPhi0 - 1 / Phi, expE = invPhi0 - 1 / Ecirc;
            sPhi[i] = log(expP);
            sE[i] = log(expE);
            logL[i] = log(Lcirc);
            const double dPdsP = Phi * Phi * expP, dEdsE = Ecirc * Ecirc * expE;
            const double dRdLv = 2 * Omega / (kappa2 * R), dLdEv = 1 / Omega;
            dRdL[i] = dRdLv * Lcirc / R;
            dLdE[i] = dLdEv * dEdsE / Lcirc;
            dPhi[i] = gR * R / dPdsP;
            if(!(Phi < 0 && gR >= 0 && (i == 0 || sPhi[i] > sPhi[i - 1])))
                throw std::runtime_error("Interpolator: potential is not monotonically increasing with radius");
            if(!(Ecirc < 0 && Lcirc >= 0 && (i == 0 || (sE[i] > sE[i - 1] && logL[i] > logL[i - 1])) && dRdLv >= 0))
                throw std::runtime_error("Interpolator: energy or angular momentum of a circular orbit are not "
                    "monotonic with radius");
            if(i == n - 1) {   // outer asymptotic behaviour
                const double num1 = 2 * gR, num2 = -R * hRR, den1 = gR, den2 = -Phi / R;
                double slope = (num1 - num2) / (den1 - den2);
                const bool roundoff =
                    fabs(num1 - num2) < fmax(fabs(num1), fabs(num2)) * ROUNDOFF_THRESHOLD ||
                    fabs(den1 - den2) < fmax(fabs(den1), fabs(den2)) * ROUNDOFF_THRESHOLD;
                if(roundoff || slope >= 0) {
                    T.slopeOut = -1; T.coefOut = 0; T.massOut = -Phi * R;
                } else {
                    if(fabs(slope + 1) < ROUNDOFF_THRESHOLD) slope = -1;
                    T.slopeOut = slope;
                    T.coefOut = (Phi + R * gR) * pow(R, -slope);
                    T.massOut = -R * Phi + T.coefOut * (slope == -1 ? log(R) : (pow(R, slope + 1) - 1) / (slope + 1));
                }
            }
        }
        pushSpline(T.lofe, sE, logL, dLdE);
        pushSpline(T.rofl, logL, logR, dRdL);
        pushSpline(T.phiofr, logR, sPhi, dPhi);
    }

    // ---- focal-distance grid in (scaled E, chi)
    const std::vector<double> gridR = interpolationGrid(Q, invPhi0, Phi0, ACCURACY_INTERP2);
    const int nE = static_cast<int>(gridR.size()), nL = SIZE_L;
    std::vector<double> gridE(nE), gridL(nL);
    const std::vector<double> v = Q.eval(gridR);
    T.gridE.resize(nE);
    T.gridL.resize(nL);
    for(int i = 0; i < nE; i++) {
        gridE[i] = v[4 * i];
        T.gridE[i] = log(invPhi0 - 1 / gridE[i]);
    }
    for(int i = 0; i < nL; i++) {
        T.gridL[i] = unscaleCub(0, 1, i / (nL - 1.), nullptr);
        gridL[i] = unscaleCub(0, 1, T.gridL[i], nullptr);
    }
    const int nNodes = (nE - 1) * (nL - 1);
    std::vector<double> nodeE(nNodes), nodeL(nNodes);
    for(int k = 0; k < nNodes; k++) { nodeE[k] = gridE[k / (nL - 1)]; nodeL[k] = gridL[k % (nL - 1)]; }
    DevBuf<double> dE, dL, dD(nNodes), dRs(nNodes);
    dE.upload(gridE);
    dL.upload(gridL);
    shellGridKernel<<<(nNodes + 31) / 32, 32>>>(P.view, nE - 1, nL - 1, dE.ptr, dL.ptr, dD.ptr, dRs.ptr);
    AGB_CUDA(cudaGetLastError());
    std::vector<double> D(nNodes);
    AGB_CUDA(cudaMemcpy(D.data(), dD.ptr, nNodes * sizeof(double), cudaMemcpyDeviceToHost));
    T.nE = nE;
    T.nL = nL;
    T.delta.assign(static_cast<size_t>(nE) * nL, 0.);
    for(int iE = 0; iE < nE - 1; iE++)
        for(int iL = 0; iL < nL - 1; iL++)
            T.delta[iE * nL + iL] = D[iE * (nL - 1) + iL];
    for(int iE = 0; iE < nE - 1; iE++) {
        T.delta[iE * nL + 0] = T.delta[iE * nL + 1];          // Lz = 0: copy the adjacent column
        T.delta[iE * nL + nL - 1] = T.delta[iE * nL + nL - 2];
    }
    for(int iL = 0; iL < nL; iL++) T.delta[(nE - 1) * nL + iL] = 0.;   // E -> 0
    for(double d : T.delta)
        if(!isFinite(d))
            throw std::runtime_error("ActionFinder: focal distance could not be computed on the grid");
    return T;
}

}  // namespace agb
