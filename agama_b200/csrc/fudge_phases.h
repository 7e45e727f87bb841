// Launchers of the phases of the Staeckel-fudge action computation (one record per point, see
// FudgeRecord): phase 1 (prepare) lives in actions.cu, phases 2 and 3 in their own units.
#pragma once
#include <cuda_runtime.h>
#include "multipole.h"
#include "fudge_types.h"

namespace agb {

struct FudgeRecord;
struct FudgeEnds;

/// half-widths of the predicted brackets, in units of the predicted fractions (order of the ROOT_*
/// kinds: nu_max, lambda_min, lambda_max)
struct BracketWidths { float w[3]; };

/// phase 2: the root searches of the integration limits, drained by a persistent grid from a
/// device work counter (8 bytes, zeroed here on the stream); with pred (n x 3 predictions) the
/// searches start on the predicted brackets; stats (4 counters, may be null) accumulates
/// searches, narrowed searches, fallbacks to the plain bracket and iterations; ends (may be null):
/// F and F' at the ends of each record's plain brackets, which the plain searches take instead of
/// evaluating them again
void launchFudgeRoots(const MultipoleView& M, long n, FudgeRecord* rec, const FudgeEnds* ends, int* iters,
    unsigned long long* counter, const float* pred, const BracketWidths& widths, unsigned long long* stats,
    cudaStream_t stream);

/// training targets of the bracket predictor from records whose plain searches are done
void launchBracketTargets(long n, const FudgeRecord* rec, float* target, float* mask, cudaStream_t stream);

/// phase 3: Jr and Jz of every valid record into act[3 i], act[3 i + 1], drained by a persistent
/// grid from a device work counter (8 bytes, zeroed here on the stream); mixed: the integrand's
/// arithmetic after F(tau) and the sums in FP32 (compensated), F(tau) in FP64
void launchFudgeIntegrals(const MultipoleView& M, const GLRules& gl, long n, const FudgeRecord* rec, double* act,
    unsigned long long* counter, bool mixed, cudaStream_t stream);

/// phase 3 with angles / frequencies: actions into act (n x 3, Jphi already there), frequencies
/// (Omega_r, Omega_z, Omega_phi) and angles (theta_r, theta_z, theta_phi) into freq / ang when
/// not null; one point per thread
void launchFudgeAngles(const MultipoleView& M, const GLRules& gl, long n, const FudgeRecord* rec, double* act,
    double* ang, double* freq, cudaStream_t stream);

}  // namespace agb
