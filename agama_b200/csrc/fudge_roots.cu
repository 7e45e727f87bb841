// Phase 2 of the Staeckel-fudge actions: the root searches of the integration limits.  In its
// own compilation unit so that its register budget does not constrain the other phases (the
// potential evaluator is a non-inlined function compiled once per unit).
#include "runtime.h"
#include "fudge.cuh"
#include "fudge_phases.h"
#include <algorithm>
#include <map>
#include <mutex>

namespace agb {

namespace {

constexpr int ROOT_BLOCK = 128;
constexpr unsigned FULL_MASK = 0xffffffffu;

/// the limit found by a plain search (nu_max falls back to |nu| when the search found no root)
__device__ __forceinline__ void storePlainLimit(FudgeRecord& r, int kind, const RootSearch& s, double u0, double nu)
{
    if(kind == ROOT_NU_MAX) r.nuMax = isFinite(s.result) ? s.result : fabs(nu);
    else if(kind == ROOT_LAMBDA_MIN) r.lambdaMin = s.result;
    else r.lambdaMax = unscaleSemiInf(u0, s.result, nullptr);
}

/// what a lane does next with its search
enum { LANE_IDLE = 0, LANE_PROPOSE = 1, LANE_EVAL = 2, LANE_VERIFY = 3 };

/** Set up a plain search on its bracket [lo, hi] with F and F' at the ends taken from phase 1
    (e may be null: the ends are then evaluated by the search): lambda_pos (shared by the lambda
    brackets), Delta^2 and |nu|; the far end of lambda_max (s = 1, lambda = inf) needs no
    evaluation either (limitRootEval's values there).  Returns LANE_IDLE when the search has
    finished at once (no sign change, or a root at an end), LANE_PROPOSE when both ends are known
    and the first iterate is due from RootSearch::propose, LANE_EVAL when *x is an end to evaluate. */
__device__ __forceinline__ int setupPlain(RootSearch& s, int kind, const FudgeEnds* e, double lo, double hi,
    double tol, double u0, double D2, double E, double* x)
{
    if(!e) { *x = s.startAbs(lo, hi, tol); return LANE_EVAL; }
    if(kind == ROOT_NU_MAX) {
        if(hi == D2) return s.setupKnownEnds(lo, hi, tol, e->fNu, e->dfNu, e->fD2, e->dfD2) ? LANE_IDLE : LANE_PROPOSE;
        *x = s.startAbs(lo, hi, tol);
        s.take(e->fNu, e->dfNu, x);         // the lower end known; the upper one is evaluated next
        return LANE_EVAL;
    }
    if(kind == ROOT_LAMBDA_MIN) {
        if(lo == D2) return s.setupKnownEnds(lo, hi, tol, e->fD2, e->dfD2, e->fPos, e->dfPos) ? LANE_IDLE : LANE_PROPOSE;
        *x = s.startKnownUpper(lo, hi, tol, e->fPos, e->dfPos);
        return LANE_EVAL;
    }
    const double fa = e->fPos / pow2(u0), da = (e->dfPos - 2 * e->fPos / u0) / pow2(u0) * u0;
    return s.setupKnownEnds(lo, hi, tol, fa, da, E, NAN) ? LANE_IDLE : LANE_PROPOSE;
}

/** The predicted bracket of a search: the predicted fraction tp -+ the half-width w (the units of
    the bracket predictor's targets), mapped to the search variable of the kind (lambda_max: the
    semi-infinite scaling about u0 = lambda_pos).  True when it lies strictly inside the plain
    bracket [lo, hi]: a prediction that reaches a plain end (limits near the focal line, or
    lambda_max far out) leaves the limit to the plain search. */
__device__ __forceinline__ bool predictedBracket(const FudgeRecord& r, int kind, double tp, double w, double u0,
    double lo, double hi, double* nlo, double* nhi)
{
    const double lmd = r.lambda - r.D2;
    if(kind == ROOT_NU_MAX) {
        const double span = r.D2 - fabs(r.nu);
        *nlo = fabs(r.nu) + (tp - w) * span;
        *nhi = fabs(r.nu) + (tp + w) * span;
    } else if(kind == ROOT_LAMBDA_MIN) {
        *nlo = r.D2 + (tp - w) * lmd;
        *nhi = r.D2 + (tp + w) * lmd;
    } else {
        const double L0 = log(fmax(r.D2 + lmd / (tp + w), u0) / u0);
        *nlo = L0 / (1 + L0);
        if(tp - w > 0) {
            const double L1 = log(fmax(r.D2 + lmd / (tp - w), u0) / u0);
            *nhi = L1 / (1 + L1);
        } else
            *nhi = hi;
    }
    return isFinite(*nlo) && isFinite(*nhi) && *nlo > lo && *nhi < hi && *nlo < *nhi;
}

/** Phase 2: every root search of the integration limits (task t = kind * n + i for the kinds
    nu_max, lambda_min, lambda_max of point i) drained from one work counter by a persistent grid.
    Each lane runs one search as a RootSearch state machine and takes the next task as soon as
    its search ends, so that the lanes of a warp meet at one potential evaluation per step instead
    of waiting for the warp's longest search.  A step of the warp has four sections, each run by
    the lanes it concerns: idle lanes take new searches and set them up; the lanes whose search
    wants its next iterate (the first one of a new search or the next one of a running search)
    propose it together; the lanes with a point evaluate F there; they feed the value to their
    search.  Proposing the iterates of new and running searches in one section keeps the
    interpolation steps of both in one instruction stream.

    With bracket predictions (pred != null: per point, in the order of the kinds, the fractions
    (nu_max - |nu|)/(D2 - |nu|), (lambda_min - D2)/(lambda - D2), (lambda - D2)/(lambda_max - D2),
    all in [0, 1]) a search runs on its plain bracket, whose end values phase 1 has evaluated, but
    its first iterate is the predicted root instead of the interpolated one (RootSearch::seed); the
    search then goes on as the plain one does and ends inside the plain bracket with the plain
    tolerance.  Seeding needs the predicted bracket (predictedBracket) strictly inside the plain
    one, and the root is accepted only if it lies inside that predicted bracket and F is negative
    half-way from it to the plain end where F is negative (one more evaluation); otherwise F may
    have more roots there and the plain search, which may end on any of them, decides.  stats (may
    be null) accumulates {searches, seeded searches, plain searches after a failed check,
    iterations} when STATS.  LEARNED = false (no predictions, no stats) compiles the plain searches
    alone, without that state and the counters (fewer registers); STATS = false leaves the
    counters out of the learned searches. */
template<bool LEARNED, bool STATS>
__global__ void __launch_bounds__(ROOT_BLOCK, 4) fudgeRootKernel(const __grid_constant__ MultipoleView M, long n,
    FudgeRecord* __restrict__ rec, const FudgeEnds* __restrict__ ends, int* __restrict__ iters,
    unsigned long long* __restrict__ counter, const float* __restrict__ pred, const BracketWidths widths,
    unsigned long long* __restrict__ stats)
{
    const long total = 3 * n;
    const unsigned lane = threadIdx.x & 31;
    bool drained = false, seeded = false, fresh = false;
    int mode = LANE_IDLE;
    long point = 0;
    int kind = 0;
    double x = 0, u0 = 0, verified = 0;
    unsigned nSearch = 0, nSeeded = 0, nFallback = 0, nIter = 0;
    FudgeFunction fnc;
    RootSearch s;
    // a plain search on the point's bracket again (after a seeded root failed its check)
    auto restartPlain = [&]() {
        const FudgeRecord& r = rec[point];
        const double lo = kind == ROOT_NU_MAX ? fabs(r.nu) : kind == ROOT_LAMBDA_MIN ? r.lambdaLower : 0;
        const double hi = kind == ROOT_NU_MAX ? r.nuUpper : kind == ROOT_LAMBDA_MIN ? r.lambdaPos : 1;
        seeded = false;
        fresh = false;
        if(STATS) nFallback++;
        mode = setupPlain(s, kind, ends ? ends + point : nullptr, lo, hi, fabs(lo - hi) * FUDGE_ACCURACY_RANGE,
                          u0, fnc.D2, fnc.E, &x);
        if(mode == LANE_IDLE) storePlainLimit(rec[point], kind, s, u0, fnc.nu);
    };
    // the search has ended with s.result: store the limit, or (a seeded search) check its root
    auto finishSearch = [&]() {
        if(STATS) nIter += s.iter;
        if(LEARNED && seeded) {
            // a seeded root is a candidate only inside the predicted bracket (it may have come from
            // another root of F in the plain bracket otherwise)
            const FudgeRecord& r = rec[point];
            const int k = kind == ROOT_NU_MAX ? 0 : kind == ROOT_LAMBDA_MIN ? 1 : 2;
            const double lo = kind == ROOT_NU_MAX ? fabs(r.nu) : kind == ROOT_LAMBDA_MIN ? r.lambdaLower : 0;
            const double hi = kind == ROOT_NU_MAX ? r.nuUpper : kind == ROOT_LAMBDA_MIN ? r.lambdaPos : 1;
            double nlo, nhi;
            predictedBracket(r, kind, pred[3 * point + k], widths.w[k], u0, lo, hi, &nlo, &nhi);
            if(isFinite(s.result) && s.result >= nlo && s.result <= nhi) {
                mode = LANE_VERIFY;
                verified = s.result;
                x = 0.5 * (s.result + (kind == ROOT_LAMBDA_MIN ? lo : hi));
            } else
                restartPlain();
            return;
        }
        mode = LANE_IDLE;
        storePlainLimit(rec[point], kind, s, u0, fnc.nu);
        if(iters) atomicAdd(iters + point, s.iter);
    };
    while(true) {
        // 1. every idle lane of the warp takes a new search (one atomic per warp and round) and
        //    sets it up
        while(true) {
            const unsigned need = __ballot_sync(FULL_MASK, mode == LANE_IDLE && !drained);
            if(!need) break;
            const int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if(static_cast<int>(lane) == leader) base = atomicAdd(counter, static_cast<unsigned long long>(__popc(need)));
            base = __shfl_sync(FULL_MASK, base, leader);
            if(mode == LANE_IDLE && !drained) {
                const long t = static_cast<long>(base) + __popc(need & ((1u << lane) - 1));
                if(t >= total) drained = true;
                else {
                    const int k = t >= 2 * n ? 2 : t >= n ? 1 : 0;      // (no 64-bit division)
                    const long i = t - k * n;
                    const FudgeRecord& r = rec[i];
                    if(r.roots & (1 << k)) {
                        point = i;
                        kind = 1 << k;
                        loadFudgeFunction(M, r, fnc);
                        u0 = r.lambdaPos;
                        const double lo = kind == ROOT_NU_MAX ? fabs(r.nu) : kind == ROOT_LAMBDA_MIN ? r.lambdaLower : 0;
                        const double hi = kind == ROOT_NU_MAX ? r.nuUpper : kind == ROOT_LAMBDA_MIN ? r.lambdaPos : 1;
                        const double tol = fabs(lo - hi) * FUDGE_ACCURACY_RANGE;
                        seeded = false;
                        mode = setupPlain(s, kind, ends ? ends + i : nullptr, lo, hi, tol, u0, r.D2, r.E, &x);
                        fresh = mode == LANE_PROPOSE;
                        if(mode == LANE_IDLE)       // no sign change or a root at an end
                            storePlainLimit(rec[i], kind, s, u0, fnc.nu);
                        if(STATS) nSearch++;
                    }
                }
            }
        }
        if(!__any_sync(FULL_MASK, mode != LANE_IDLE)) break;
        // 2. the next iterate of every search that wants one: the first of a new search (replaced
        //    by the predicted root when the prediction is usable) or the next of a running one
        if(mode == LANE_PROPOSE) {
            if(s.propose(&x))
                finishSearch();
            else {
                mode = LANE_EVAL;
                if(LEARNED && pred && fresh) {
                    // points predicted near the focal line (nu_max or lambda_min within two
                    // bracket half-widths of D2) keep the plain searches for all limits:
                    // there the GL action integrals resolve the integrands poorly and depend
                    // on the limits to the last bits of the plain searches
                    const FudgeRecord& r = rec[point];
                    const int k = kind == ROOT_NU_MAX ? 0 : kind == ROOT_LAMBDA_MIN ? 1 : 2;
                    const bool nearFocal = pred[3 * point] + 2 * widths.w[0] >= 1 ||
                                           pred[3 * point + 1] - 2 * widths.w[1] <= 0;
                    const double lo = kind == ROOT_NU_MAX ? fabs(r.nu) : kind == ROOT_LAMBDA_MIN ? r.lambdaLower : 0;
                    const double hi = kind == ROOT_NU_MAX ? r.nuUpper : kind == ROOT_LAMBDA_MIN ? r.lambdaPos : 1;
                    double nlo, nhi;
                    if(!nearFocal && predictedBracket(r, kind, pred[3 * point + k], widths.w[k], u0, lo, hi, &nlo, &nhi)) {
                        const double tp = pred[3 * point + k], lmd = r.lambda - r.D2;
                        double guess;
                        if(kind == ROOT_NU_MAX) guess = fabs(r.nu) + tp * (r.D2 - fabs(r.nu));
                        else if(kind == ROOT_LAMBDA_MIN) guess = r.D2 + tp * lmd;
                        else {          // in the semi-infinite scaling about lambda_pos
                            const double L0 = log(fmax(r.D2 + lmd / tp, u0) / u0);
                            guess = L0 / (1 + L0);
                        }
                        if(isFinite(guess)) seeded = s.seed(guess, &x);
                    }
                    if(STATS) nSeeded += seeded;
                }
            }
            fresh = false;
        }
        // 3. F (and F') at the points of the lanes that have one
        double fx = 0, dx = 0;
        if(mode == LANE_EVAL || mode == LANE_VERIFY) limitRootEval(fnc, kind, u0, x, &fx, &dx);
        // 4. the values fed to the searches
        if(mode == LANE_EVAL) {
            const int r = s.take(fx, dx, &x);
            if(r == 0) finishSearch();
            else mode = r == 1 ? LANE_PROPOSE : LANE_EVAL;
        } else if(LEARNED && mode == LANE_VERIFY) {
            // a root from a seeded search: F must have the sign of the plain bracket's end
            // half-way between the root and that end (lambda_max: towards infinity in the
            // scaled variable; lambda_min: towards D2; nu_max: towards D2), where it is
            // negative; otherwise F has more roots there and the plain search decides
            if(STATS) nIter++;
            if(fx < 0) {
                mode = LANE_IDLE;
                FudgeRecord& w = rec[point];
                if(kind == ROOT_NU_MAX) w.nuMax = verified;
                else if(kind == ROOT_LAMBDA_MIN) w.lambdaMin = verified;
                else w.lambdaMax = unscaleSemiInf(u0, verified, nullptr);
                if(iters) atomicAdd(iters + point, s.iter + 1);
            } else
                restartPlain();
        }
    }
    if(STATS && stats) {       // one atomic per warp and counter
        nSearch = __reduce_add_sync(FULL_MASK, nSearch);
        nSeeded = __reduce_add_sync(FULL_MASK, nSeeded);
        nFallback = __reduce_add_sync(FULL_MASK, nFallback);
        nIter = __reduce_add_sync(FULL_MASK, nIter);
        if(lane == 0) {
            atomicAdd(stats, static_cast<unsigned long long>(nSearch));
            atomicAdd(stats + 1, static_cast<unsigned long long>(nSeeded));
            atomicAdd(stats + 2, static_cast<unsigned long long>(nFallback));
            atomicAdd(stats + 3, static_cast<unsigned long long>(nIter));
        }
    }
}

/// bracket-predictor training targets of the records (after the plain searches), as described at
/// fudgeRootKernel, and a 0/1 mask of the searched limits
__global__ void bracketTargetKernel(long n, const FudgeRecord* __restrict__ rec, float* __restrict__ target,
    float* __restrict__ mask)
{
    const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if(i >= n) return;
    const FudgeRecord r = rec[i];
    const double lmd = r.lambda - r.D2, span = r.D2 - fabs(r.nu);
    const double t[3] = { (r.nuMax - fabs(r.nu)) / span, (r.lambdaMin - r.D2) / lmd, lmd / (r.lambdaMax - r.D2) };
    for(int k = 0; k < 3; k++) {
        const bool ok = r.valid && (r.roots & (1 << k)) && isFinite(t[k]);
        target[3 * i + k] = ok ? static_cast<float>(t[k]) : 0.f;
        mask[3 * i + k] = ok ? 1.f : 0.f;
    }
}

/// resident blocks of a root-kernel variant on the current device (cached per device and variant)
template<bool LEARNED, bool STATS>
int rootGridSize()
{
    static std::mutex mutex;
    static std::map<int, int> cache;
    int dev;
    AGB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mutex);
    auto it = cache.find(dev);
    if(it != cache.end()) return it->second;
    int sms = 0, perSM = 0;
    AGB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    AGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fudgeRootKernel<LEARNED, STATS>, ROOT_BLOCK, 0));
    const int grid = std::max(1, sms * std::max(1, perSM));
    cache[dev] = grid;
    return grid;
}

}  // namespace

void launchFudgeRoots(const MultipoleView& M, long n, FudgeRecord* rec, const FudgeEnds* ends, int* iters,
    unsigned long long* counter, const float* pred, const BracketWidths& widths, unsigned long long* stats,
    cudaStream_t stream)
{
    if(n <= 0) return;
    AGB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), stream));
    const long tasks = (3 * n + ROOT_BLOCK - 1) / ROOT_BLOCK;
    if(stats) {              // learned or plain searches with the counters
        const long grid = std::min<long>(rootGridSize<true, true>(), tasks);
        fudgeRootKernel<true, true><<<grid, ROOT_BLOCK, 0, stream>>>(M, n, rec, ends, iters, counter, pred, widths, stats);
    } else if(pred) {
        const long grid = std::min<long>(rootGridSize<true, false>(), tasks);
        fudgeRootKernel<true, false><<<grid, ROOT_BLOCK, 0, stream>>>(M, n, rec, ends, iters, counter, pred, widths,
            nullptr);
    } else {
        const long grid = std::min<long>(rootGridSize<false, false>(), tasks);
        fudgeRootKernel<false, false><<<grid, ROOT_BLOCK, 0, stream>>>(M, n, rec, ends, iters, counter, nullptr, widths,
            nullptr);
    }
    AGB_CUDA(cudaGetLastError());
}

void launchBracketTargets(long n, const FudgeRecord* rec, float* target, float* mask, cudaStream_t stream)
{
    if(n <= 0) return;
    bracketTargetKernel<<<(n + 255) / 256, 256, 0, stream>>>(n, rec, target, mask);
    AGB_CUDA(cudaGetLastError());
}

}  // namespace agb
