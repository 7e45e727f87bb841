// DOP853 orbit integration kernels and their host launchers.
//
// Reference: orbit::BaseOrbitIntegrator::run (src/orbit.cpp:52-84), OrbitIntegrator<Car>::init
// (:98-117) and OdeStepperDOP853::init / initTimeStep / doStep (src/math_ode.cpp:35-406).
// Each thread integrates one orbit; the stage vectors k2..k10 live in shared memory laid out
// [vector][component][thread] so that a warp touches 32 consecutive doubles per access.
// A batch is either mapped one orbit per thread, or drained from a device work queue (an
// atomic counter) by a grid sized to the GPU, which balances orbits of very different length.
#include "runtime.h"
#include "dop853.cuh"
#include "host_pipeline.h"
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <algorithm>
#include <set>
#include <utility>
#include <vector>

namespace agb {

namespace {

constexpr int ORBIT_BLOCK_MAX = 128;                 // largest block of the orbit kernels
constexpr int NUM_STAGE_VECTORS = 9;                 // k2 .. k10 (k11..k13 reuse k2..k4)
constexpr int MAX_ATTEMPTS_PER_STEP = 1000;          // guard against a runaway rejection loop
constexpr double HMIN = 1e-12, HMAX = 1e12;          // initial-step limits, src/math_ode.cpp:40

struct StageStore {
    double* base;
    int stride;                                      // = blockDim.x
    __device__ double& at(int v, int c) const { return base[(v * 6 + c) * stride]; }
};

/// The Runge-Kutta stages of one DOP853 attempt as table rows: row r forms the point of stage
/// r+2 (k_{r+2}) as x + h sum coef * k_src, row 11 the 8th-order solution (weights b).  Sources:
/// -1 = k1 (registers), otherwise a stage slot; results go to slot dest[r].  Terms and their order
/// are those of OdeStepperDOP853::doStep (src/math_ode.cpp:243-300); unused terms have coef 0.
constexpr int NUM_ROWS = 12, MAX_TERMS = 9, K1 = -1;
struct StageTable {
    double coef[NUM_ROWS][MAX_TERMS];
    double c[NUM_ROWS];
    signed char src[NUM_ROWS][MAX_TERMS];
    signed char dest[NUM_ROWS];
};

__host__ __device__ constexpr StageTable makeStageTable()
{
    using namespace dp853;
    StageTable T{};
    const double coef[NUM_ROWS][MAX_TERMS] = {
        { a21 },
        { a31, a32 },
        { a41, a43 },
        { a51, a53, a54 },
        { a61, a64, a65 },
        { a71, a74, a75, a76 },
        { a81, a84, a85, a86, a87 },
        { a91, a94, a95, a96, a97, a98 },
        { a101, a104, a105, a106, a107, a108, a109 },
        { a111, a114, a115, a116, a117, a118, a119, a1110 },
        { a121, a124, a125, a126, a127, a128, a129, a1210, a1211 },
        { b1, b6, b7, b8, b9, b10, b11, b12 } };
    const signed char src[NUM_ROWS][MAX_TERMS] = {
        { K1 }, { K1, 0 }, { K1, 1 }, { K1, 1, 2 }, { K1, 2, 3 }, { K1, 2, 3, 4 }, { K1, 2, 3, 4, 5 },
        { K1, 2, 3, 4, 5, 6 }, { K1, 2, 3, 4, 5, 6, 7 }, { K1, 2, 3, 4, 5, 6, 7, 8 },
        { K1, 2, 3, 4, 5, 6, 7, 8, 0 }, { K1, 4, 5, 6, 7, 8, 0, 1 } };
    const int nterms[NUM_ROWS] = { 1, 2, 2, 3, 3, 4, 5, 6, 7, 8, 9, 8 };
    const double c[NUM_ROWS] = { c2, c3, c4, c5, c6, c7, c8, c9, c10, c11, 1, 1 };
    const signed char dest[NUM_ROWS] = { 0, 1, 2, 3, 4, 5, 6, 7, 8, 0, 1, -1 };
    for(int r = 0; r < NUM_ROWS; r++) {
        for(int t = 0; t < MAX_TERMS; t++) {
            T.coef[r][t] = t < nterms[r] ? coef[r][t] : 0;
            T.src[r][t] = t < nterms[r] ? src[r][t] : K1;
        }
        T.c[r] = c[r];
        T.dest[r] = dest[r];
    }
    return T;
}
__constant__ StageTable STAGE_TABLE = makeStageTable();

/** The 7th-order dense output of the last accepted step [t, t + h] at offset (0..h) from its start
    (OdeStepperDOP853::getSol and its coefficients, src/math_ode.cpp:381-426), in the integration
    (inertial) frame. */
__device__ void denseOutput(double h, double offset, const double* x, const double* xt, const double* k1,
    const double* k13, const StageStore& S, double* v)
{
    using namespace dp853;
    if(offset == h) {
        for(int c = 0; c < 6; c++) v[c] = xt[c];
        return;
    }
    if(offset == 0) {
        for(int c = 0; c < 6; c++) v[c] = x[c];
        return;
    }
    const double p = offset / h, q = 1.0 - p;
    for(int c = 0; c < 6; c++) {
        const double k6 = S.at(4, c), k7 = S.at(5, c), k8 = S.at(6, c), k9 = S.at(7, c), k10 = S.at(8, c),
            k11 = S.at(0, c), k12 = S.at(1, c);
        const double xd = xt[c] - x[c], xc = h * k1[c] - xd;
        const double r4 = xd - h * k13[c] - xc;
        const double r5 = h * (d41 * k1[c] + d46 * k6 + d47 * k7 + d48 * k8 + d49 * k9 + d410 * k10 +
                               d411 * k11 + d412 * k12 + d413 * k13[c]);
        const double r6 = h * (d51 * k1[c] + d56 * k6 + d57 * k7 + d58 * k8 + d59 * k9 + d510 * k10 +
                               d511 * k11 + d512 * k12 + d513 * k13[c]);
        const double r7 = h * (d61 * k1[c] + d66 * k6 + d67 * k7 + d68 * k8 + d69 * k9 + d610 * k10 +
                               d611 * k11 + d612 * k12 + d613 * k13[c]);
        const double r8 = h * (d71 * k1[c] + d76 * k6 + d77 * k7 + d78 * k8 + d79 * k9 + d710 * k10 +
                               d711 * k11);
        v[c] = x[c] + p * (xd + q * (xc + p * (r4 + q * (r5 + p * (r6 + q * (r7 + p * r8))))));
    }
}

/// a phase-space point of the integration frame rotated to the frame of the potential at time
/// tabs (OrbitIntegrator<Car>::getSolNative, src/orbit.cpp:119-133)
__device__ __forceinline__ void toPotentialFrame(double Omega, double tabs, const double* v, double* o)
{
    double ca = 1, sa = 0;
    if(Omega != 0) sincos(Omega * tabs, &sa, &ca);
    o[0] = v[0] * ca + v[1] * sa;
    o[1] = v[1] * ca - v[0] * sa;
    o[2] = v[2];
    o[3] = v[3] * ca + v[4] * sa;
    o[4] = v[4] * ca - v[3] * sa;
    o[5] = v[5];
}

/** Trajectory samples inside one accepted step [t, t + h] at the regular times k T/(trajSize-1)
    (RuntimeTrajectory::processTimestep, src/orbit.cpp:15-47: sample range with the 10 eps
    round-off allowance, offsets clipped into the step) from the dense output of the step, rotated
    to the frame of the potential at each sample time. */
__device__ void sampleStep(const OrbitParams& P, long i, double tEnd, double sign, double t, double h,
    const double* x, const double* xt, const double* k1, const double* k13, const StageStore& S)
{
    const double dt = fabs(tEnd) / (P.trajSize - 1), tend = t + h;
    const double roundoff = 10 * DBL_EPSILON * fmax(fabs(tend), fabs(t));
    long iout = static_cast<long>(ceil(sign * t / dt));
    long iend = static_cast<long>((sign * tend + roundoff) / dt);
    if(iend > P.trajSize - 1) iend = P.trajSize - 1;
    for(; iout <= iend; iout++) {
        const double timeout = sign * dt * iout;
        const double offset = clip(sign * (timeout - t), 0.0, sign * h) * sign;
        double v[6];
        denseOutput(h, offset, x, xt, k1, k13, S, v);
        toPotentialFrame(P.Omega, t + offset, v, P.traj + (i * P.trajSize + iout) * 6);
    }
}

/// samples of one accepted step for the target of the batch (RuntimeFncTarget::processTimestep,
/// src/galaxymodel_target.h:140-152): NUM_SAMPLES_PER_STEP points at the middles of equal
/// sub-steps of the step, each weighted by the sub-step's duration
constexpr int TARGET_SAMPLES_PER_STEP = 10;
__device__ void targetStep(const OrbitParams& P, long i, double t, double h, const double* x, const double* xt,
    const double* k1, const double* k13, const StageStore& S)
{
    const double substep = h / TARGET_SAMPLES_PER_STEP;
    double* row = P.target.datacube + i * P.target.numValues;
    for(int k = 0; k < TARGET_SAMPLES_PER_STEP; k++) {
        const double off = substep * (k + 0.5);
        double v[6], w[6];
        denseOutput(h, off, x, xt, k1, k13, S, v);
        toPotentialFrame(P.Omega, t + off, v, w);
        targetAddPoint(P.target, w, substep, row);
    }
}

/// phases of the per-lane integration state machine
enum { PH_FETCH, PH_INIT1, PH_INIT2, PH_INIT3, PH_STAGE, PH_FINISH };

/** One orbit per lane, driven as a state machine around ONE call of the right-hand side per
    loop iteration: lanes of a warp at different stages, attempts, orbits or in the initial-step
    estimate all meet at that call, instead of serialising at twelve separate call sites.  The
    step algorithm (OdeStepperDOP853::initTimeStep / doStep and the run loop of
    BaseOrbitIntegrator::run, src/math_ode.cpp:35-406, src/orbit.cpp:52-84) is unchanged:
    initial step from Euler and Heun probes, error norm err5 |h| / sqrt(6 (err5 + 0.01 err3))
    weighted by (accAbs + accRel max|x|) accFac, accept at err <= 1, step factor
    min(finc, safe / err^(1/8)), rejection with the nbad counter; the final point is rotated
    to the frame of the potential at time tb + hLast (RuntimeTrajectory semantics).
    queue != nullptr: lanes take orbits from the work counter until it passes n; otherwise lane
    i integrates orbit i only.
    G > 1: a group of G consecutive lanes integrates one orbit: every lane of the group runs the
    same state machine on the same data (the group's sums are bit-identical in all its lanes, so
    its control flow never splits) and the lanes share the spline evaluations of each right-hand
    side; lane 0 of the group takes the orbits from the counter and writes the results.
    MIXED: the forces of the multi-harmonic kind with the m != 0 harmonics in FP32 (the radial m = 0
    part, the Fourier sums, the state, the stages and the error norm stay FP64). */
template<int KIND, int G, bool MIXED>
__global__ void __launch_bounds__(ORBIT_BLOCK_MAX) dop853Kernel(const __grid_constant__ MultipoleView M, const OrbitParams P,
    long n, const double* __restrict__ ic, const double* __restrict__ T, double* __restrict__ out,
    long* __restrict__ nsteps, long* __restrict__ nrej, int* __restrict__ status,
    unsigned long long* queue)
{
    const int gl = threadIdx.x % G;
    const unsigned gmask = groupMask<G>();
    using namespace dp853;
    extern __shared__ double smem[];
    __shared__ StageTable tab;
    for(int k = threadIdx.x; k < static_cast<int>(sizeof(StageTable) / sizeof(double)); k += blockDim.x)
        reinterpret_cast<double*>(&tab)[k] = reinterpret_cast<const double*>(&STAGE_TABLE)[k];
    __syncthreads();
    const StageStore S{ smem + threadIdx.x, static_cast<int>(blockDim.x) };
    const double Om = P.Omega;

    long i = queue ? -1 : (blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x) / G;
    if(!queue && i >= n) return;
    int phase = queue ? PH_FETCH : PH_INIT1;
    double x[6], k1[6], xt[6], k1b[6];
    double t = 0, tEnd = 0, sign = 1, h = 0, h1 = 0, hNext = 0, accFac = 1, preverr = INFINITY, tb = 0, hLast = 0,
        remaining = 0, targetTime = 0;
    long steps = 0, rejects = 0;
    int st = ORBIT_OK, row = 0, nbad = 0, attempts = 0;

    // begin an attempt with the current h (zero, non-finite or endlessly rejected: give up)
    auto startAttempt = [&]() {
        if(h == 0 || !isFinite(h) || ++attempts > MAX_ATTEMPTS_PER_STEP) { st = ORBIT_BAD_STEP; phase = PH_FINISH; return; }
        row = 0;
        phase = PH_STAGE;
    };
    // begin the next step, or finish the orbit when the end time is reached
    auto startStep = [&]() {
        if(t == tEnd) { phase = PH_FINISH; return; }
        remaining = tEnd - t;
        h = fmin(remaining * sign, hNext) * sign;
        nbad = 0; attempts = 0; preverr = INFINITY;
        startAttempt();
    };

    while(true) {
        if(phase == PH_FETCH) {
            long v = 0;
            if(gl == 0) v = static_cast<long>(atomicAdd(queue, 1ull));
            i = G > 1 ? static_cast<long>(__shfl_sync(gmask, static_cast<unsigned long long>(v), 0, G)) : v;
            if(i >= n) break;
            phase = PH_INIT1;
        }
        if(phase == PH_INIT1) {          // a new orbit: load its start
            for(int c = 0; c < 6; c++) x[c] = ic[6 * i + c];
            tEnd = T[i];
            t = 0; tb = 0; hLast = 0; steps = 0; rejects = 0; st = ORBIT_OK; accFac = 1; targetTime = 0;
            sign = tEnd >= 0 ? 1 : -1;
            if(P.traj && gl == 0) {
                // no sample yet; an orbit that is not integrated gets its start as sample 0 (and, for
                // T = 0, as sample 1 too: the reference's zero sampling interval records the start
                // and the end of its single zero step)
                double* o = P.traj + i * P.trajSize * 6;
                for(int k = 0; k < P.trajSize * 6; k++) o[k] = NAN;
                if(tEnd == 0 || !isFinite(tEnd))
                    for(int k = 0; k < (tEnd == 0 ? 2 : 1) && k < P.trajSize; k++)
                        for(int c = 0; c < 6; c++) o[6 * k + c] = x[c];
            }
        }
        if(phase == PH_FINISH) {
            if(gl == 0) {
                double ca = 1, sa = 0;
                if(Om != 0) sincos(Om * (hLast + tb), &sa, &ca);
                out[6 * i + 0] = x[0] * ca + x[1] * sa;
                out[6 * i + 1] = x[1] * ca - x[0] * sa;
                out[6 * i + 2] = x[2];
                out[6 * i + 3] = x[3] * ca + x[4] * sa;
                out[6 * i + 4] = x[4] * ca - x[3] * sa;
                out[6 * i + 5] = x[5];
                if(nsteps) nsteps[i] = steps;
                if(nrej) nrej[i] = rejects;
                if(status) status[i] = st;
                if(P.target.degree >= 0) {
                    // RuntimeFncTarget's finalisation: the sums converted to FP32, then scaled
                    // by the inverse integration time in FP32 (src/galaxymodel_target.h:127-135)
                    const double* row = P.target.datacube + i * P.target.numValues;
                    float* o = P.target.output + i * P.target.numValues;
                    const float inv = static_cast<float>(1. / targetTime);
                    for(int k = 0; k < P.target.numValues; k++) {
                        o[k] = static_cast<float>(row[k]);
                        if(targetTime != 0) o[k] *= inv;
                    }
                }
            }
            if(!queue) break;
            phase = PH_FETCH;
            continue;
        }
        // ---- the point at which the right-hand side is wanted
        double tt;
        if(phase == PH_INIT1) {
            tt = t;
            for(int c = 0; c < 6; c++) xt[c] = x[c];
        } else if(phase == PH_INIT2) {
            tt = t + h1;
            for(int c = 0; c < 6; c++) xt[c] = x[c] + h1 * k1[c];
        } else if(phase == PH_INIT3) {
            tt = t + h1;
            for(int c = 0; c < 6; c++) xt[c] = x[c] + 0.5 * h1 * (k1[c] + S.at(0, c));
        } else {
            tt = t + tab.c[row] * h;     // c = 1 for k12 and the 8th-order point: t + h
            for(int c = 0; c < 6; c++) {
                double acc = tab.coef[row][0] * k1[c];
                for(int m = 1; m < MAX_TERMS; m++) {
                    const int sl = tab.src[row][m];
                    acc += tab.coef[row][m] * (sl < 0 ? k1[c] : S.at(sl, c));
                }
                if(row == NUM_ROWS - 1) k1b[c] = acc;
                xt[c] = x[c] + h * acc;
            }
        }
        // ---- the one evaluation site
        const bool wantAcc = phase == PH_INIT1 || (phase == PH_STAGE && row == NUM_ROWS - 1);
        double k[6], af = 1;
        orbitRHS<3, KIND, G, MIXED>(M, Om, tt, xt, k, wantAcc ? &af : nullptr);
        // ---- use the result
        if(phase == PH_INIT1) {
            for(int c = 0; c < 6; c++) k1[c] = k[c];
            accFac = af;
            if(tEnd == 0 || !isFinite(tEnd)) { phase = PH_FINISH; continue; }
            double nx = 0, nd = 0;
            for(int c = 0; c < 6; c++) { nx += x[c] * x[c]; nd += k1[c] * k1[c]; }
            h1 = fmax(HMIN, fmin(HMAX, sqrt(nx / nd) * 0.01));
            phase = PH_INIT2;
        } else if(phase == PH_INIT2) {
            for(int c = 0; c < 6; c++) S.at(0, c) = k[c];
            phase = PH_INIT3;
        } else if(phase == PH_INIT3) {
            // initTimeStep (src/math_ode.cpp:35-91): Euler + Heun probes, Aarseth-like estimate
            double h2 = INFINITY;
            for(int c = 0; c < 6; c++) {
                const double k2c = S.at(0, c);
                const double d0 = fmax(P.accAbs, fmax(fabs(x[c]), fabs(xt[c])));
                const double d1 = fmax(fabs(k1[c]), fabs(k[c]));
                const double d2 = fabs((3 * k2c - k1[c] - 2 * k[c]) / h1);
                const double d3 = fabs(6 * (k[c] - k2c) / (h1 * h1));
                h2 = fmin(h2, (d0 * d2 + d1 * d1) / (d1 * d3 + d2 * d2));
            }
            hNext = fmax(HMIN, fmin(HMAX, pow(P.accRel, 1. / 8) * sqrt(h2))) * accFac;
            startStep();
        } else if(row < NUM_ROWS - 1) {
            const int d = tab.dest[row];
            for(int c = 0; c < 6; c++) S.at(d, c) = k[c];
            row++;
        } else {
            // ---- error estimate (3rd and 5th order embedded solutions), k13 = k
            double err5 = 0, err3 = 0;
            for(int c = 0; c < 6; c++) {
                const double sk = (P.accAbs + P.accRel * fmax(fabs(x[c]), fabs(xt[c]))) * af;
                if(sk == 0) continue;
                err3 += pow2((k1b[c] - bhh1 * k1[c] - bhh2 * S.at(7, c) - bhh3 * S.at(1, c)) / sk);
                err5 += pow2((er1 * k1[c] + er6 * S.at(4, c) + er7 * S.at(5, c) + er8 * S.at(6, c) +
                    er9 * S.at(7, c) + er10 * S.at(8, c) + er11 * S.at(0, c) + er12 * S.at(1, c)) / sk);
            }
            const double den = sqrt(6 * (err5 + 0.01 * err3));
            const double err = den == 0 ? 0 : err5 * fabs(h) / den;
            if(!isFinite(err)) { st = ORBIT_NONFINITE; phase = PH_FINISH; continue; }
            double fac = sqrt(sqrt(sqrt(err)));
            bool accepted = false;
            if(err <= 1) {
                hNext = fabs(h) * fmin(finc, safe / fac);
                accepted = true;
            } else {
                if(err > 0.5 * preverr) {
                    nbad++;
                    if(nbad >= 2) fac = 1 / fdec;
                    if(nbad >= 4) { hNext = fabs(h); accepted = true; }
                } else
                    nbad = 0;
                if(!accepted) {
                    preverr = err;
                    h *= fmax(fdec, safe / fac);
                    rejects++;
                    startAttempt();
                    continue;
                }
            }
            if(P.traj && gl == 0) sampleStep(P, i, tEnd, sign, t, h, x, xt, k1, k, S);
            if(P.target.degree >= 0 && gl == 0) {
                targetStep(P, i, t, h, x, xt, k1, k, S);
                targetTime += h;
            }
            for(int c = 0; c < 6; c++) { x[c] = xt[c]; k1[c] = k[c]; }
            tb = t;
            hLast = h;
            t = h == remaining ? tEnd : t + h;
            if(++steps >= P.maxSteps) {
                if(t != tEnd) st = ORBIT_MAX_STEPS;
                phase = PH_FINISH;
                continue;
            }
            startStep();
        }
    }
}

}  // namespace

size_t orbitSharedBytes(int block) { return sizeof(double) * NUM_STAGE_VECTORS * 6 * block; }

namespace {

using OrbitKernel = void (*)(const MultipoleView, const OrbitParams, long, const double*, const double*, double*,
    long*, long*, int*, unsigned long long*);

OrbitKernel orbitKernel(int kind, int lanes, bool mixed)
{
    if(kind == EVAL_FAST) {
        if(mixed) return dop853Kernel<EVAL_FAST, 1, true>;
        switch(lanes) {
            case 2: return dop853Kernel<EVAL_FAST, 2, false>;
            case 4: return dop853Kernel<EVAL_FAST, 4, false>;
            case 8: return dop853Kernel<EVAL_FAST, 8, false>;
            default: return dop853Kernel<EVAL_FAST, 1, false>;
        }
    }
    return kind == EVAL_AXI ? dop853Kernel<EVAL_AXI, 1, false> : dop853Kernel<EVAL_GENERAL, 1, false>;
}

/// FP32 non-axisymmetric harmonics in later batches (multi-harmonic potentials only; off by default)
std::atomic<int> g_mixedSetting{ 0 };

/// raise the dynamic shared-memory limit of an orbit kernel on the current device once (the
/// stage vectors of 128 threads take 54 KB, above the default 48 KB)
void allowOrbitSharedMemory(OrbitKernel kernel)
{
    static std::mutex mutex;
    static std::set<std::pair<int, const void*>> done;
    int dev;
    AGB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mutex);
    const auto key = std::make_pair(dev, reinterpret_cast<const void*>(kernel));
    if(done.count(key)) return;
    AGB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
        static_cast<int>(orbitSharedBytes(ORBIT_BLOCK_MAX))));
    done.insert(key);
}

void launchOrbitKernel(const MultipoleView& M, const OrbitParams& P, long n, const double* ic, const double* T,
    double* out, long* nsteps, long* nrej, int* status, unsigned long long* queue, int lanes, int block, bool mixed,
    cudaStream_t stream)
{
    if(block != 32 && block != 64 && block != 128) block = 64;
    const size_t shmem = orbitSharedBytes(block);
    mixed = mixed && evalKindOf(M) == EVAL_FAST;
    if(mixed) lanes = 1;
    const OrbitKernel kernel = orbitKernel(evalKindOf(M), lanes, mixed);
    allowOrbitSharedMemory(kernel);
    const long threads = n * lanes;
    long grid;
    if(queue) {
        int dev, sms, perSM = 0;
        AGB_CUDA(cudaGetDevice(&dev));
        AGB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        AGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, block, shmem));
        grid = static_cast<long>(sms) * (perSM > 0 ? perSM : 1);
        const long needed = (threads + block - 1) / block;
        if(grid > needed) grid = needed;
        AGB_CUDA(cudaMemsetAsync(queue, 0, sizeof(unsigned long long), stream));
    } else {
        grid = (threads + block - 1) / block;
    }
    kernel<<<grid, block, shmem, stream>>>(M, P, n, ic, T, out, nsteps, nrej, status, queue);
    AGB_CUDA(cudaGetLastError());
}

}  // namespace

// ------------------------------------------------------------------------------------------
// Launch shape (lanes per orbit and threads per block): chosen by a timing trial on the caller's
// own orbits, once per device, potential, batch-size class (powers of two) and precision, then
// cached.  Every shape gives the same bits (the lanes of a group sum the harmonics in one order;
// the block size only changes which orbits share a block), so the choice never changes a result.

namespace {

std::mutex g_shapeMutex;
std::map<std::tuple<int, const void*, int, int>, OrbitShape> g_shapeChoice;
std::atomic<int> g_laneSetting{ 0 }, g_blockSetting{ 0 };
constexpr int TRIAL_ORBITS = 32768, TRIAL_STEPS = 24;

/// time each candidate shape on the first orbits of the batch, each integrated for TRIAL_STEPS
/// steps; candidates: lanes in {1, 2, 4, 8} (the multi-harmonic kind in FP64; 1 otherwise) times
/// blocks in {32, 64, 128}
OrbitShape tuneShape(const MultipoleView& M, const OrbitParams& P, long n, const double* ic, const double* T,
    bool mixed, int fixedLanes, int fixedBlock, cudaStream_t stream)
{
    const long m = std::min<long>(n, TRIAL_ORBITS);
    OrbitParams Pt = P;
    Pt.maxSteps = TRIAL_STEPS;
    Pt.traj = nullptr;
    Pt.trajSize = 0;
    Pt.target = TargetView();
    Scratch scratch(m * 6 * sizeof(double) + 256, stream);
    double* out = static_cast<double*>(scratch.ptr);
    unsigned long long* counter = reinterpret_cast<unsigned long long*>(out + 6 * m);
    std::vector<int> laneList, blockList;
    const bool groups = evalKindOf(M) == EVAL_FAST && !mixed;
    for(int l : { 1, 2, 4, 8 })
        if((fixedLanes ? l == fixedLanes : true) && (groups || l == 1)) laneList.push_back(l);
    for(int b : { 32, 64, 128 })
        if(fixedBlock ? b == fixedBlock : true) blockList.push_back(b);
    if(laneList.empty()) laneList.push_back(1);
    if(blockList.empty()) blockList.push_back(64);
    cudaEvent_t a, b;
    AGB_CUDA(cudaEventCreate(&a));
    AGB_CUDA(cudaEventCreate(&b));
    OrbitShape best;
    best.lanes = laneList[0];
    best.block = blockList[0];
    float bestMs = INFINITY;
    // one untimed run absorbs the one-time set-up (module loading, attributes)
    launchOrbitKernel(M, Pt, m, ic, T, out, nullptr, nullptr, nullptr, counter, laneList[0], blockList[0], mixed, stream);
    for(int l : laneList) {
        for(int bl : blockList) {
            AGB_CUDA(cudaEventRecord(a, stream));
            launchOrbitKernel(M, Pt, m, ic, T, out, nullptr, nullptr, nullptr, counter, l, bl, mixed, stream);
            AGB_CUDA(cudaEventRecord(b, stream));
            AGB_CUDA(cudaEventSynchronize(b));
            float ms = 0;
            AGB_CUDA(cudaEventElapsedTime(&ms, a, b));
            if(ms < bestMs) { bestMs = ms; best.lanes = l; best.block = bl; }
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return best;
}

}  // namespace

void setOrbitLanes(int lanes) { g_laneSetting = lanes; }
void setOrbitBlock(int block) { g_blockSetting = block; }
void setOrbitMixedPrecision(bool mixed) { g_mixedSetting = mixed ? 1 : 0; }

OrbitShape orbitShapeFor(const MultipoleView& M, const OrbitParams& P, long n, const double* ic, const double* T,
    cudaStream_t stream)
{
    const bool mixed = g_mixedSetting != 0 && evalKindOf(M) == EVAL_FAST;
    const bool groups = evalKindOf(M) == EVAL_FAST && !mixed;
    int fixedLanes = g_laneSetting, fixedBlock = g_blockSetting;
    if(fixedLanes != 1 && fixedLanes != 2 && fixedLanes != 4 && fixedLanes != 8) fixedLanes = 0;
    if(!groups) fixedLanes = 1;
    if(fixedBlock != 32 && fixedBlock != 64 && fixedBlock != 128) fixedBlock = 0;
    if(fixedLanes && fixedBlock) { OrbitShape s; s.lanes = fixedLanes; s.block = fixedBlock; return s; }
    int dev;
    AGB_CUDA(cudaGetDevice(&dev));
    int bucket = 0;
    while((1L << bucket) < n) bucket++;
    // the key holds the fixed parts too (0 = tuned), so fixing one of them tunes only the other
    const auto key = std::make_tuple(dev, static_cast<const void*>(M.spl2d), bucket,
        (mixed ? 1 : 0) | (fixedLanes << 1) | (fixedBlock << 5));
    {
        std::lock_guard<std::mutex> lock(g_shapeMutex);
        auto it = g_shapeChoice.find(key);
        if(it != g_shapeChoice.end()) return it->second;
    }
    const OrbitShape shape = tuneShape(M, P, n, ic, T, mixed, fixedLanes, fixedBlock, stream);
    std::lock_guard<std::mutex> lock(g_shapeMutex);
    g_shapeChoice[key] = shape;
    return shape;
}

void launchOrbits(const MultipoleView& M, const OrbitParams& P, long n, const double* ic, const double* T,
    double* out, long* nsteps, long* nrej, int* status, unsigned long long* queue, cudaStream_t stream, OrbitShape shape)
{
    if(n <= 0) return;
    if(shape.lanes <= 0 || shape.block <= 0) shape = orbitShapeFor(M, P, n, ic, T, stream);
    launchOrbitKernel(M, P, n, ic, T, out, nsteps, nrej, status, queue, shape.lanes, shape.block,
        g_mixedSetting != 0, stream);
}

// ------------------------------------------------------------------------------------------
// Work-queue orbit integration without any allocation by the library.
//
// Some callers cannot have a library allocate device memory: applications whose own memory
// manager has reserved (nearly) all of the GPU's memory up front, so a cudaMalloc fails or
// fragments their pool; latency-critical loops in which cudaMalloc / cudaFree would synchronise
// the device and stall the caller's other streams; and plugin hosts that account for all device
// memory and forbid libraries from allocating behind their back.  For them the work-queue
// counters live in a fixed static array in device memory, loaded with the library (every GPU
// that loads it holds these 256 bytes until the process exits).

/// number of independent work-queue counters (one per batch that may run at the same time)
constexpr int NOALLOC_QUEUE_SLOTS = 32;

/// the counters; each call clears its own slot on its stream before the launch
static __device__ __align__(256) unsigned long long g_noallocQueue[NOALLOC_QUEUE_SLOTS];

namespace {
std::mutex g_noallocMutex;
std::map<int, unsigned long long*> g_noallocAddress;   // device address of the array, per device
}

int noallocQueueSlots() { return NOALLOC_QUEUE_SLOTS; }

void launchOrbitsNoAlloc(const MultipoleView& M, const OrbitParams& P, long n, const double* ic, const double* T,
    double* out, long* nsteps, long* nrej, int* status, int slot, cudaStream_t stream)
{
    if(slot < 0 || slot >= NOALLOC_QUEUE_SLOTS)
        throw std::invalid_argument("integrateOrbitsManyDeviceNoAlloc: queueSlot must be in 0.." +
            std::to_string(NOALLOC_QUEUE_SLOTS - 1) + " (the static work-queue array has " +
            std::to_string(NOALLOC_QUEUE_SLOTS) + " counters)");
    int dev;
    AGB_CUDA(cudaGetDevice(&dev));
    unsigned long long* base = nullptr;
    {
        // one-time set-up per device, with that device current: the host-side name of a
        // __device__ array is not a device address, so look the address up once and cache it
        std::lock_guard<std::mutex> lock(g_noallocMutex);
        auto it = g_noallocAddress.find(dev);
        if(it == g_noallocAddress.end()) {
            AGB_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&base), g_noallocQueue));
            g_noallocAddress[dev] = base;
        } else
            base = it->second;
    }
    // the launch clears the counter (cudaMemsetAsync on the stream) before the kernel runs;
    // one lane per orbit (the lane autotuner's trial would allocate scratch), always FP64
    if(n <= 0) return;
    launchOrbitKernel(M, P, n, ic, T, out, nsteps, nrej, status, base + slot, 1, 64, false, stream);
}

}  // namespace agb
