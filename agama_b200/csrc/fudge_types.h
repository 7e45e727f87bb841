// Plain data shared by the host runtime and the fudge device code.
#pragma once
#include <vector>

namespace agb {

constexpr int GL_MAX_ORDER = 40;                 // reference MAX_GL_ORDER, src/math_core.h:577

/// Gauss-Legendre rules on [0, 1] for the orders the reference tabulates (1..20, 25, 32, 40):
/// nodes and weights of rule n start at offset[n]; orders without a rule map to the next one
struct GLRules {
    int offset[GL_MAX_ORDER + 1];   // -1 where no rule
    const double* nodes;
    const double* weights;
};

/// 1-D quintic spline stored as [x | f | f' | f''] with n nodes each
struct Spline1dView { int n; const double* t; };

/// focal-distance table and the L_circ(E) interpolator of an action finder (device view)
struct FudgeTables {
    double invPhi0;               // 1 / Phi(0) of the finder
    int nE, nL;                   // Delta(scaledE, chi) table
    const double* gridE;
    const double* gridL;
    const double* delta;          // [nE][nL]
    double iInvPhi0, slopeOut, coefOut, massOut;   // potential::Interpolator scalars
    Spline1dView LofE, RofL, PhiofR;
};

/// host copy of the same tables: the focal-distance grid of ActionFinderAxisymFudge
/// (src/actions_staeckel.cpp:751-795) and the potential::Interpolator pieces used by L_circ(E)
struct FinderTablesHost {
    double invPhi0 = 0, interpInvPhi0 = 0, slopeOut = -1, coefOut = 0, massOut = 0;
    int nE = 0, nL = 0;
    std::vector<double> gridE, gridL, delta;        // scaled E, chi = s(Lz/Lcirc), Delta [nE][nL]
    std::vector<double> lofe, rofl, phiofr;         // [x | f | f' | f''] each
};

}  // namespace agb
