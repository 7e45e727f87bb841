// Multipole potential: host-side description of the tables and the flat, pointer-based
// view of them that device code receives by value.
//
// The potential is the reference's potential::Multipole (src/potential_multipole.h:206-304):
// inside [r_min(1+eps^(1/3)), r_max(1-eps^(1/3))] it is a set of 2-D quintic splines in
// (ln r, tau = z/(r+R)), one per azimuthal harmonic m (lmax > 2), or 1-D quintic splines in
// ln r for each (l,m) coefficient (lmax <= 2); outside, two power-law asymptotic expansions.
#pragma once
#include <vector>
#include <string>
#include <map>
#include "common.cuh"

namespace agb {

/// symmetry flags (values of coord::SymmetryType, reference src/coord.h:50-75)
enum Symmetry {
    SYM_NONE = 0, SYM_XREFL = 1, SYM_YREFL = 2, SYM_ZREFL = 4, SYM_REFL = 8,
    SYM_ZROT = 16, SYM_ROT = 32,
    SYM_TRIAXIAL = 15, SYM_AXISYMMETRIC = 31, SYM_SPHERICAL = 63
};

/** The set of non-trivial (l,m) terms of a spherical-harmonic expansion and their order;
    reference math::SphHarmIndices, src/math_sphharm.cpp:156-230. */
struct HarmIndices {
    int lmax = 0, mmax = 0, step = 1, sym = SYM_SPHERICAL;
    int lminArr[2 * LMAX_MAX + 1];   // for m = -mmax..mmax
    AGB_HD int lmin(int m) const { return (m >= -mmax && m <= mmax) ? lminArr[m + mmax] : lmax + 1; }
    AGB_HD int mmin() const { return (sym & SYM_YREFL) == SYM_YREFL ? 0 : -mmax; }
    AGB_HD static int index(int l, int m) { return l * (l + 1) + m; }
    AGB_HD int size() const { return (lmax + 1) * (lmax + 1); }
};

/// device view of one power-law asymptotic expansion (inner or outer)
struct PowerLawView {
    HarmIndices ind;
    double r0sq;          // square of the matching radius
    int inner;            // 1: inner (v = l), 0: outer (v = -l-1)
    double Q;             // extra r^2 term of the inner monopole
    const double* S;      // slopes, (lmax+1)^2
    const double* U;      // amplitudes of (r/r0)^s
    const double* W;      // amplitudes of (r/r0)^v
};

/// device view of a complete Multipole potential
struct MultipoleView {
    HarmIndices ind;
    int is2d;             // 1: per-m 2-D splines; 0: per-(l,m) 1-D splines (lmax <= 2)
    double rInnerSq, rOuterSq;   // squared switching radii to the asymptotic expansions
    int nr; const double* lnr;   // radial grid in ln r
    int nt; const double* tau;   // angular grid in tau (2-D case)
    const double* lnrInvH;       // 1 / (lnr[k+1] - lnr[k]), k < nr - 1 (correctly rounded)
    const double* tauInvH;       // 1 / (tau[j+1] - tau[j]), j < nt - 1
    double lnrScale, tauScale;   // (n - 1) / (grid[n-1] - grid[0]): binSearchScaled's first guess
    int splSlot[2 * LMAX_MAX + 1];  // slot of the 2-D spline for m (index m+mmax), -1 if empty
    const double* spl2d;  // [slot][nr][nt][NODE_STRIDE]: f fx fy fxx fxy fyy fxxy fxyy fxxyy pad
    const float* spl2d32; // the same table rounded to FP32 (mixed-precision evaluation of m != 0)
    const double* spl1d;  // [c][nr][3]: f f' f''  (1-D case; all (lmax+1)^2 coefficients)
    int logScaling;
    double invPhi0;
    PowerLawView inner, outer;
    /// the non-empty harmonics for the register-resident evaluator: m = 0 first, then the others
    /// by ascending m; nFast = 0 when there are more than FAST_MAX_HARMONICS of them
    int nFast;
    int fastM[FAST_MAX_HARMONICS];
    int fastSlot[FAST_MAX_HARMONICS];
};

/** Host-side Multipole: owns the tables built from the radial grid and the coefficients
    Phi_lm(r_k), dPhi_lm/dr(r_k), exactly as the reference constructor
    Multipole(gridRadii, Phi, dPhi) does (src/potential_multipole.cpp:1491-1516). */
struct MultipoleHost {
    HarmIndices ind;
    int is2d = 0;
    std::vector<double> radii, lnr, tau;
    int splSlot[2 * LMAX_MAX + 1];
    int numSlots = 0;
    std::vector<double> spl2d, spl1d;
    int logScaling = 0;
    double invPhi0 = 0;
    struct Asympt { HarmIndices ind; double r0sq = 0, Q = 0; int inner = 0; std::vector<double> S, U, W; };
    Asympt inner, outer;
    // original coefficients (kept for export)
    std::vector<std::vector<double>> Phi, dPhi;
};

/// build the tables; throws std::invalid_argument / std::runtime_error on bad input
MultipoleHost buildMultipole(const std::vector<double>& radii,
    const std::vector<std::vector<double>>& Phi, const std::vector<std::vector<double>>& dPhi);

/// parse the reference's Multipole coefficient text format (written by writePotential,
/// reference src/potential_factory.cpp:909-930, read at :725-746)
void readMultipoleCoefFile(const std::string& fileName, std::vector<double>& radii,
    std::vector<std::vector<double>>& Phi, std::vector<std::vector<double>>& dPhi);

/// write the coefficients in the same text format (the layout of writePotentialMultipole,
/// reference src/potential_factory.cpp:909-930: [Potential] section, gridSizeR, lmax, symmetry
/// name, #Phi and #dPhi/dr blocks of tab-separated columns l=..,m=..), with every number in 17
/// significant digits so that reading the file back gives the same doubles
void writeMultipoleCoefFile(const std::string& fileName, const std::vector<double>& radii,
    const std::vector<std::vector<double>>& Phi, const std::vector<std::vector<double>>& dPhi, int symmetry);

/** the coefficients of a Multipole built from density models (the Poisson solve of the
    reference's createMultipole, src/potential_multipole.cpp:1400-1441): densities = key=value
    parameters of each component (type, mass, scaleRadius, ...; summed), params = the Multipole's
    own (lmax, mmax, gridSizeR, rmin, rmax, symmetry, fixOrder); keys in lower case */
void multipoleCoefsFromDensity(const std::vector<std::map<std::string, std::string>>& densities,
    const std::map<std::string, std::string>& params, std::vector<double>& radii,
    std::vector<std::vector<double>>& Phi, std::vector<std::vector<double>>& dPhi);

// helpers shared with the action-finder construction
double lambertW(double x, bool lowerBranch);
void glNodesWeights(int n, double* nodes, double* weights);   // on [-1, 1], ascending
std::vector<double> quinticSecondDerivs(const std::vector<double>& x, const std::vector<double>& f,
    const std::vector<double>& fder);
HarmIndices makeIndices(int lmax, int mmax, int sym);
HarmIndices indicesFromCoefs(const std::vector<double>& D);

}  // namespace agb
