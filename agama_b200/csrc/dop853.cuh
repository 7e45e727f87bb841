// DOP853 orbit integration on the device: one orbit per thread, Runge-Kutta stage vectors in
// shared memory (thread-interleaved, bank-conflict free), state and step control in registers.
#pragma once
#include "multipole_eval.cuh"

namespace agb {

/** A runtime function of the orbits: time-weighted samples of each orbit accumulated into the
    basis elements of a spheroidal density grid (the reference's RuntimeFncTarget with
    TargetDensityClassic<N>, src/galaxymodel_target.h:99-150, src/galaxymodel_densitygrid.cpp:149-237):
    shells in the spheroidal radius sqrt((x/ax)^2 + (y/ay)^2 + (z/az)^2), each octant surface cut
    into three panes of strips x strips cells; degree 0 = top-hat cells, 1 = trilinear nodes. */
struct TargetView {
    int degree = -1;              ///< -1: no target; 0: DensityClassicTopHat; 1: DensityClassicLinear
    int strips = 0, nShells = 0, valuesPerShell = 0, numValues = 0;
    const double* shellRadii = nullptr;   ///< nShells positive increasing radii
    double axisX = 1, axisY = 1, axisZ = 1;
    double* datacube = nullptr;   ///< n x numValues accumulators (zeroed before the launch)
    float* output = nullptr;      ///< n x numValues results, normalised by the integration time
};

/// integration parameters shared by all orbits of a batch
struct OrbitParams {
    double Omega;        ///< pattern speed of the rotating frame
    double accRel;       ///< relative accuracy (DOP853 "accuracy")
    double accAbs;       ///< absolute accuracy (0 in the reference's orbit integrator)
    long   maxSteps;     ///< maximum number of accepted steps per orbit
    int    trajSize = 0; ///< samples per orbit at regular times 0 .. T (0: final point only)
    double* traj = nullptr;   ///< n x trajSize x 6 samples (rotating frame), NaN where none
    TargetView target;        ///< optional runtime function of the orbits (degree -1: none)
};

/** Add one point to the basis elements of a classic density grid, weighted by mult
    (TargetDensityClassic<N>::addPoint and getCornerIndicesClassic, src/galaxymodel_densitygrid.cpp:59-84,
    :170-238): the shell from a binary search in the spheroidal radius, the pane from the largest
    coordinate, the strips from the angles atan(c1/c0), atan(c2/c0) in units of pi/4.  Points
    outside the last shell add nothing; a point whose pane cannot be determined (NaN coordinates,
    where the reference throws) adds nothing either.  values is the row of one orbit, owned by one
    lane: the sums run in the order of the samples, as in the reference. */
__device__ inline void targetAddPoint(const TargetView& T, const double p[3], double mult, double* values)
{
    const double X = fabs(p[0] / T.axisX), Y = fabs(p[1]) / T.axisY, Z = fabs(p[2]) / T.axisZ;
    const double r = sqrt(X * X + Y * Y + Z * Z);
    const int indShell = binSearch(r, T.shellRadii, T.nShells) + 1;
    if(indShell >= T.nShells || mult == 0) return;
    int pane;
    double c0, c1, c2;
    if(X >= Y && X > Z)       { pane = 0; c0 = X; c1 = Y; c2 = Z; }
    else if(Y >= Z && Y > X)  { pane = 1; c0 = Y; c1 = Z; c2 = X; }
    else if(Z >= X && Z >= Y) { pane = 2; c0 = Z; c1 = X; c2 = Y; }
    else return;
    const int S = T.strips;
    double ratio1 = fmin(atan(c1 / c0) * (4 / M_PI), 1.) * S;
    double ratio2 = fmin(atan(c2 / c0) * (4 / M_PI), 1.) * S;
    const int ind1 = min(static_cast<int>(ratio1), S - 1), ind2 = min(static_cast<int>(ratio2), S - 1);
    if(T.degree == 0) {
        values[ind1 + (ind2 + pane * S) * S + indShell * T.valuesPerShell] += mult;
        return;
    }
    // degree 1: the four corner nodes of the cell on the two shells around the point
    const int ll = ind1 + (ind2 + pane * S) * (S + 1), ul = ll + 1;
    int lu, uu;
    if(ind2 < S - 1) { lu = ll + S + 1; uu = lu + 1; }
    else {
        const int adj = (pane + 2) % 3;
        lu = (ind1 + adj * S + 1) * (S + 1) - 1;
        uu = ind1 < S - 1 ? lu + S + 1 : 3 * S * (S + 1);
    }
    ratio1 -= ind1;
    ratio2 -= ind2;
    double val = indShell == 0 ? mult * r / T.shellRadii[0] :
        mult * (r - T.shellRadii[indShell - 1]) / (T.shellRadii[indShell] - T.shellRadii[indShell - 1]);
    double* off = values + indShell * T.valuesPerShell + 1;
    off[ll] += (1 - ratio1) * (1 - ratio2) * val;
    off[ul] += ratio1 * (1 - ratio2) * val;
    off[lu] += (1 - ratio1) * ratio2 * val;
    off[uu] += ratio1 * ratio2 * val;
    if(indShell == 0)
        values[0] += mult - val;
    else {
        off -= T.valuesPerShell;
        val = mult - val;
        off[ll] += (1 - ratio1) * (1 - ratio2) * val;
        off[ul] += ratio1 * (1 - ratio2) * val;
        off[lu] += (1 - ratio1) * ratio2 * val;
        off[uu] += ratio1 * ratio2 * val;
    }
}

/// per-orbit outcome codes
enum OrbitStatus { ORBIT_OK = 0, ORBIT_MAX_STEPS = 1, ORBIT_BAD_STEP = 2, ORBIT_NONFINITE = 3, ORBIT_BUDGET = 4 };

// Coefficients of the 8(5,3) Dormand-Prince pair (Hairer, Norsett & Wanner, "Solving ODEs I",
// DOP853), the same tableau as the reference's OdeStepperDOP853 (src/math_ode.cpp:112-237).
namespace dp853 {
constexpr double c2 = 0.05260015195876773187856, c3 = 0.07890022793815159781784,
    c4 = 0.11835034190722739672676, c5 = 0.28164965809277260327324, c6 = 0.33333333333333333333333,
    c7 = 0.25, c8 = 0.30769230769230769230769, c9 = 0.65128205128205128205128, c10 = 0.6,
    c11 = 0.85714285714285714285714;
constexpr double a21 = 0.05260015195876773187856;
constexpr double a31 = 0.01972505698453789945446, a32 = 0.05917517095361369836338;
constexpr double a41 = 0.02958758547680684918169, a43 = 0.08876275643042054754507;
constexpr double a51 = 0.24136513415926668550237, a53 = -0.88454947932828608534486,
    a54 = 0.92483400326179200311574;
constexpr double a61 = 0.03703703703703703703704, a64 = 0.17082860872947387127960,
    a65 = 0.12546768756682242501669;
constexpr double a71 = 0.037109375, a74 = 0.17025221101954403931498, a75 = 0.06021653898045596068502,
    a76 = -0.017578125;
constexpr double a81 = 0.03709200011850479271088, a84 = 0.17038392571223999381021,
    a85 = 0.10726203044637328465181, a86 = -0.01531943774862440175279, a87 = 0.00827378916381402288758;
constexpr double a91 = 0.62411095871607571711443, a94 = -3.36089262944694129406857,
    a95 = -0.86821934684172600681819, a96 = 27.5920996994467083049416, a97 = 20.1540675504778934086187,
    a98 = -43.4898841810699588477366;
constexpr double a101 = 0.47766253643826436589043, a104 = -2.48811461997166764192642,
    a105 = -0.59029082683684299637145, a106 = 21.2300514481811942347289, a107 = 15.2792336328824235832597,
    a108 = -33.2882109689848629194453, a109 = -0.02033120170850862613582;
constexpr double a111 = -0.93714243008598732571704, a114 = 5.18637242884406370830024,
    a115 = 1.09143734899672957818500, a116 = -8.14978701074692612513997, a117 = -18.5200656599969598641566,
    a118 = 22.7394870993505042818970, a119 = 2.49360555267965238987089, a1110 = -3.04676447189821950038237;
constexpr double a121 = 2.27331014751653820792360, a124 = -10.5344954667372501984067,
    a125 = -2.00087205822486249909676, a126 = -17.9589318631187989172766, a127 = 27.9488845294199600508500,
    a128 = -2.85899827713502369474066, a129 = -8.87285693353062954433549, a1210 = 12.3605671757943030647266,
    a1211 = 0.64339274601576353035597;
constexpr double b1 = 0.05429373411656876223805, b6 = 4.45031289275240888144114, b7 = 1.89151789931450038304282,
    b8 = -5.80120396001058478146721, b9 = 0.31116436695781989440892, b10 = -0.15216094966251607855618,
    b11 = 0.20136540080403034837478, b12 = 0.04471061572777259051769;
constexpr double bhh1 = 0.24409448818897637795276, bhh2 = 0.73384668828161185734136,
    bhh3 = 0.02205882352941176470588;
constexpr double er1 = 0.01312004499419488073250, er6 = -1.22515644637620444072057,
    er7 = -0.49575894965725019152141, er8 = 1.66437718245498653696153, er9 = -0.35032884874997368168865,
    er10 = 0.33417911871301747902973, er11 = 0.08192320648511571246571, er12 = -0.02235530786388629525884;
// 7th-order dense output (the reference's variant of the interpolant, src/math_ode.cpp:196-233)
constexpr double d41 = -5.40685903845352664250302, d46 = 367.268892700041893590281,
    d47 = 154.609958204083905482676, d48 = -505.920283865412564024766, d49 = 15.5975154819608130688200,
    d410 = -26.1936204184402805956691, d411 = -0.74003512364122230844721, d412 = 1.11776539319431476294221,
    d413 = -0.33333333333333333333333;
constexpr double d51 = 6.51987095363079615048119, d56 = -1066.34956011730205278592,
    d57 = -351.864047514639508625601, d58 = 1363.51955696662884408368, d59 = -112.727669432657582669864,
    d510 = 159.796191868560289612921, d511 = -2.13865100308788816220259, d512 = -3.75569172113289760348584,
    d513 = 7.0;
constexpr double d61 = 10.4698004763293477204238, d66 = -1380.01473607038123167155,
    d67 = -531.219827862514074379012, d68 = 1866.98964341870892451324, d69 = -53.3302605020547902574560,
    d610 = 82.4147560258671369782481, d611 = 7.38443654502992069572676, d612 = 0.41729908012587751149843,
    d613 = -3.11111111111111111111111;
constexpr double d71 = -16.6338582677165354330709, d76 = 4516.16568914956011730205,
    d77 = 1393.85185384057776465219, d78 = -5687.52042419481539670071, d79 = 473.965563750151263163661,
    d710 = -661.810776942355889724311, d711 = -18.0180473354013232598119;
constexpr double fdec = 0.333, finc = 6.0, safe = 0.9;   // step-size control
}  // namespace dp853

/** Right-hand side of the orbit ODE in the inertial frame with the potential rotating at
    Omega: dx/dt = v, dv/dt = -R(-Omega t) grad Phi(R(Omega t) x); optionally the accuracy factor
    min(1, |E| / max(|Phi|, K)).  Reference OrbitIntegrator<Car>::eval, src/orbit.cpp:183-208.
    G > 1: called together by a group of G lanes with the same point, which share the spline
    evaluations (the multi-harmonic evaluator kind only). */
template<int NQ, int KIND, int G = 1, bool MIXED = false>
__device__ __forceinline__ void orbitRHS(const MultipoleView& M, double Omega, double time,
    const double* xv, double* dxdt, double* accFac)
{
    double ca = 1, sa = 0;
    if(Omega != 0) sincos(Omega * time, &sa, &ca);
    double Epot, g[3], h[6];
    evalMultipoleCar<NQ, KIND, G, MIXED>(M, xv[0] * ca + xv[1] * sa, xv[1] * ca - xv[0] * sa, xv[2], &Epot, g, h);
    dxdt[0] = xv[3];
    dxdt[1] = xv[4];
    dxdt[2] = xv[5];
    dxdt[3] = -g[0] * ca + g[1] * sa;
    dxdt[4] = -g[1] * ca - g[0] * sa;
    dxdt[5] = -g[2];
    if(accFac) {
        const double Ekin = 0.5 * (xv[3] * xv[3] + xv[4] * xv[4] + xv[5] * xv[5]);
        *accFac = fmin(1., fabs(Epot + Ekin) / fmax(fabs(Epot), Ekin));
    }
}

}  // namespace agb
