// Staeckel-fudge action kernels, the device-resident action finder and their host launchers.
#include "runtime.h"
#include <array>
#include <mutex>
#include <atomic>
#include <vector>
#include "fudge.cuh"
#include "host_pipeline.h"
#include "fudge_phases.h"
#include "mlp.h"
#include <algorithm>
#include <mutex>
#include <map>

namespace agb {

namespace {

/// Gauss-Legendre rules on [0,1] for the orders 1..20, 25, 32, 40 (the set the reference
/// tabulates, src/math_glquadrature.h), computed by Newton iteration in extended precision
struct GLRulesHost { int offset[GL_MAX_ORDER + 1]; std::vector<double> nodes, weights; };

GLRulesHost makeGLRules()
{
    GLRulesHost g;
    for(int n = 0; n <= GL_MAX_ORDER; n++) g.offset[n] = -1;
    const int orders[] = { 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 25, 32, 40 };
    for(int n : orders) {
        g.offset[n] = static_cast<int>(g.nodes.size());
        std::vector<long double> x(n), w(n);
        for(int i = 0; i < n; i++) {
            long double t = cosl(3.14159265358979323846264338327950288L * (i + 0.75L) / (n + 0.5L)), dp = 1;
            for(int it = 0; it < 100; it++) {
                long double p0 = 1, p1 = t;
                for(int k = 2; k <= n; k++) { long double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
                if(n == 1) { p1 = t; p0 = 1; }
                dp = n * (t * p1 - p0) / (t * t - 1);
                const long double dx = p1 / dp;
                t -= dx;
                if(fabsl(dx) < 1e-19L) break;
            }
            long double p0 = 1, p1 = t;
            for(int k = 2; k <= n; k++) { long double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
            if(n == 1) { p1 = t; p0 = 1; }
            dp = n * (t * p1 - p0) / (t * t - 1);
            x[i] = (1 - t) / 2;                    // ascending nodes on [0, 1]
            w[i] = 1 / ((1 - t * t) * dp * dp);    // = (2 / ((1-t^2) P'^2)) / 2
        }
        for(int i = 0; i < n; i++) { g.nodes.push_back(static_cast<double>(x[i])); g.weights.push_back(static_cast<double>(w[i])); }
    }
    return g;
}

/// per-device copy of the quadrature rules (uploaded on first use)
struct GLDevice { DevBuf<double> nodes, weights; GLRules view; };
std::mutex g_glMutex;
std::map<int, GLDevice*> g_gl;

const GLRules& glRulesForCurrentDevice()
{
    int dev;
    AGB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_glMutex);
    auto it = g_gl.find(dev);
    if(it != g_gl.end()) return it->second->view;
    static const GLRulesHost host = makeGLRules();
    GLDevice* d = new GLDevice;
    d->nodes.upload(host.nodes);
    d->weights.upload(host.weights);
    for(int n = 0; n <= GL_MAX_ORDER; n++) d->view.offset[n] = host.offset[n];
    d->view.nodes = d->nodes.ptr;
    d->view.weights = d->weights.ptr;
    g_gl[dev] = d;
    return d->view;
}

constexpr int PREPARE_BLOCK = 128;
constexpr long POINTS_PER_PASS = 1L << 20;     // records of one pass: 128 MB of scratch

/// Phase 1, one point per thread: cylindrical coordinates, potential, focal distance (FINDER:
/// from the finder's table; otherwise fd[i], or fd0 if fd is null), integrals of motion, the
/// limits that need no root search and the brackets of those that do -> one record per point.
/// Jphi (and NaN Jr, Jz of points without actions) are written directly.  Optional outputs:
/// Delta used, root-finder iterations (zeroed here, counted by phase 2).  ends[i]: F and F' at the
/// ends of the record's plain root brackets, for the root searches.
template<bool FINDER>
__global__ void __launch_bounds__(PREPARE_BLOCK, 5) fudgePrepareKernel(const __grid_constant__ MultipoleView M,
    const __grid_constant__ FudgeTables F, long n, const double* __restrict__ posvel, const double* __restrict__ fd,
    double fd0, FudgeRecord* __restrict__ rec, double* __restrict__ act, double* __restrict__ fdOut,
    int* __restrict__ iters, float* __restrict__ features, FudgeEnds* __restrict__ ends)
{
    const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if(i >= n) return;
    double w[6], pc[6];
    for(int c = 0; c < 6; c++) w[c] = posvel[6 * i + c];
    carToCylPosVel(w, pc);
    double Phi;
    CylDerivs g; CylHess h;
    evalMultipoleCylCall<1, EVAL_AXI>(M, pc[0], pc[1], 0, &Phi, &g, &h);   // axisymmetric: no azimuth
    const double delta = FINDER ? finderFocalDistance(F, pc, Phi) : (fd ? fd[i] : fd0);
    FudgeRecord r;
    double a[3];
    FudgeEnds e;
    fudgePrepare(M, pc, Phi, delta, r, a, &e);
    rec[i] = r;
    if(r.valid) ends[i] = e;
    act[3 * i + 2] = a[2];
    if(!r.valid) { act[3 * i] = a[0]; act[3 * i + 1] = a[1]; }
    if(fdOut) fdOut[i] = delta;
    if(iters) iters[i] = 0;
    if(features) {
        // inputs of the bracket predictor: the point's (R, z, vR, vz, vphi) with E and Lz in
        // scale-free form -- ln r, |z| / r, velocities over the escape speed sqrt(-2 Phi) (so
        // that E = Phi (1 - v^2 / v_esc^2) and Lz = R vphi follow), ln(Delta / r); symmetric
        // under z -> -z and Lz -> -Lz like the limits themselves
        const double r = fmax(sqrt(pc[0] * pc[0] + pc[1] * pc[1]), 1e-300), vesc = sqrt(fmax(-2 * Phi, 1e-300));
        const float f[6] = { static_cast<float>(log(r)), static_cast<float>(fabs(pc[1]) / r),
            static_cast<float>(pc[3] / vesc), static_cast<float>((pc[1] >= 0 ? pc[4] : -pc[4]) / vesc),
            static_cast<float>(fabs(pc[5]) / vesc), static_cast<float>(log(fmax(delta, 1e-300) / r)) };
        for(int k = 0; k < 6; k++) features[6 * i + k] = f[k];
    }
}

/// Optional timing of the phases: while on, every pass records CUDA events on its stream before
/// and after each phase (prepare, bracket inference, root searches, integrals); the durations are
/// read and summed when the timing is switched off.
struct PhaseTimer {
    std::mutex mutex;
    bool on = false;
    std::vector<std::array<cudaEvent_t, 5>> passes;
};
PhaseTimer g_phaseTimer;

/// mixed-precision action integrals in later calls (off by default)
std::atomic<int> g_actionMixed{ 0 };

/// events of one pass, or null when the timing is off
std::array<cudaEvent_t, 5>* phaseEvents()
{
    std::lock_guard<std::mutex> lock(g_phaseTimer.mutex);
    if(!g_phaseTimer.on) return nullptr;
    std::array<cudaEvent_t, 5> ev;
    for(auto& e : ev) AGB_CUDA(cudaEventCreate(&e));
    g_phaseTimer.passes.push_back(ev);
    return &g_phaseTimer.passes.back();
}

/// the three phases over passes of at most POINTS_PER_PASS points (bounded scratch); with ang or
/// freq the last phase also computes angles / frequencies (act may then be null).  With a
/// bracket predictor (bp), phase 1 also writes its inputs and the root searches start on its
/// predictions; with samples, phase 3 is replaced by the predictor's training targets.
template<bool FINDER>
void runActions(const MultipoleView& M, const FudgeTables& F, long n, const double* posvel, const double* fd,
    double fd0, double* act, double* ang, double* freq, double* fdOut, int* iters, const BracketPlan* bp,
    const BracketSamples* samples, cudaStream_t stream)
{
    if(n <= 0) return;
    const GLRules& gl = glRulesForCurrentDevice();
    const long pass = std::min(n, POINTS_PER_PASS);
    const bool predict = bp && bp->net;
    // records, two work counters, the actions of a pass when the caller wants none, and the
    // predictor's inputs and outputs
    const size_t recBytes = pass * (sizeof(FudgeRecord) + sizeof(FudgeEnds)) + 256;
    const size_t actBytes = act ? 0 : pass * 3 * sizeof(double);
    const size_t featBytes = (predict ? pass * 9 * sizeof(float) : 0) + 256;
    Scratch scratch(recBytes + actBytes + featBytes, stream);
    FudgeRecord* rec = static_cast<FudgeRecord*>(scratch.ptr);
    FudgeEnds* ends = reinterpret_cast<FudgeEnds*>(rec + pass);
    unsigned long long* counter = reinterpret_cast<unsigned long long*>(ends + pass);
    double* actTmp = reinterpret_cast<double*>(static_cast<char*>(scratch.ptr) + recBytes);
    float* feat = predict ? reinterpret_cast<float*>(static_cast<char*>(scratch.ptr) + recBytes + actBytes) : nullptr;
    float* pred = predict ? feat + pass * 6 : nullptr;
    const bool angles = ang || freq;
    BracketWidths widths{ { 0, 0, 0 } };
    if(predict) for(int k = 0; k < 3; k++) widths.w[k] = bp->widths[k];
    for(long first = 0; first < n; first += pass) {
        const long count = std::min(pass, n - first);
        std::array<cudaEvent_t, 5> ev;
        bool timed = false;
        if(auto* e = phaseEvents()) { ev = *e; timed = true; }
        auto mark = [&](int k) { if(timed) AGB_CUDA(cudaEventRecord(ev[k], stream)); };
        mark(0);
        int* it = iters ? iters + first : nullptr;
        double* a = act ? act + 3 * first : actTmp;
        float* f = samples ? samples->features + 6 * first : feat;
        fudgePrepareKernel<FINDER><<<(count + PREPARE_BLOCK - 1) / PREPARE_BLOCK, PREPARE_BLOCK, 0, stream>>>(
            M, F, count, posvel + 6 * first, fd ? fd + first : nullptr, fd0, rec, a,
            fdOut ? fdOut + first : nullptr, it, f, ends);
        AGB_CUDA(cudaGetLastError());
        mark(1);
        if(predict) bp->net->predict(count, feat, pred, stream);
        mark(2);
        launchFudgeRoots(M, count, rec, ends, it, counter, pred, widths, bp ? bp->stats : nullptr, stream);
        mark(3);
        if(samples)
            launchBracketTargets(count, rec, samples->target + 3 * first, samples->mask + 3 * first, stream);
        else if(angles)
            launchFudgeAngles(M, gl, count, rec, a, ang ? ang + 3 * first : nullptr,
                freq ? freq + 3 * first : nullptr, stream);
        else
            launchFudgeIntegrals(M, gl, count, rec, a, counter + 1, g_actionMixed != 0, stream);
        mark(4);
    }
}

}  // namespace

void setActionMixedPrecision(bool mixed) { g_actionMixed = mixed ? 1 : 0; }

void setActionPhaseTiming(bool on, double* ms, long* passes)
{
    std::lock_guard<std::mutex> lock(g_phaseTimer.mutex);
    if(!on) {
        double sum[4] = { 0, 0, 0, 0 };
        for(auto& ev : g_phaseTimer.passes) {
            AGB_CUDA(cudaEventSynchronize(ev[4]));
            for(int k = 0; k < 4; k++) {
                float t = 0;
                AGB_CUDA(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
                sum[k] += t;
            }
        }
        if(ms) for(int k = 0; k < 4; k++) ms[k] = sum[k];
        if(passes) *passes = static_cast<long>(g_phaseTimer.passes.size());
    }
    for(auto& ev : g_phaseTimer.passes)
        for(auto& e : ev) cudaEventDestroy(e);
    g_phaseTimer.passes.clear();
    g_phaseTimer.on = on;
}

void launchActionsFixedDelta(const MultipoleView& M, long n, const double* posvel, const double* fd, double fd0,
    double* act, double* ang, double* freq, int* iters, cudaStream_t stream)
{
    FudgeTables dummy{};
    runActions<false>(M, dummy, n, posvel, fd, fd0, act, ang, freq, nullptr, iters, nullptr, nullptr, stream);
}

void launchActionsFinder(const MultipoleView& M, const FudgeTables& F, long n, const double* posvel,
    double* act, double* ang, double* freq, double* fdOut, int* iters, cudaStream_t stream, const BracketPlan* bp)
{
    runActions<true>(M, F, n, posvel, nullptr, 0, act, ang, freq, fdOut, iters, bp, nullptr, stream);
}

void launchBracketSamples(const MultipoleView& M, const FudgeTables& F, long n, const double* posvel,
    const BracketSamples& samples, cudaStream_t stream)
{
    runActions<true>(M, F, n, posvel, nullptr, 0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, &samples, stream);
}

// ------------------------------------------------------------------------------------------

DeviceActionFinder::~DeviceActionFinder() { delete brackets; }

DeviceActionFinder* createDeviceActionFinder(DevicePotential* pot, const FinderTablesHost& T)
{
    if(!pot->axisymmetric)
        throw std::invalid_argument("Fudge approximation only works for axisymmetric potentials");
    if(T.nE < 2 || T.nL < 2 || T.gridE.size() != static_cast<size_t>(T.nE) ||
        T.gridL.size() != static_cast<size_t>(T.nL) || T.delta.size() != static_cast<size_t>(T.nE * T.nL) ||
        T.lofe.size() % 4 || T.rofl.size() % 4 || T.phiofr.size() % 4)
        throw std::invalid_argument("ActionFinder: inconsistent table sizes");
    DeviceActionFinder* A = new DeviceActionFinder;
    A->pot = pot;
    A->host = T;
    A->gridE.upload(T.gridE);
    A->gridL.upload(T.gridL);
    A->delta.upload(T.delta);
    A->lofe.upload(T.lofe);
    A->rofl.upload(T.rofl);
    A->phiofr.upload(T.phiofr);
    FudgeTables& F = A->view;
    F.invPhi0 = T.invPhi0;
    F.nE = T.nE; F.nL = T.nL;
    F.gridE = A->gridE.ptr; F.gridL = A->gridL.ptr; F.delta = A->delta.ptr;
    F.iInvPhi0 = T.interpInvPhi0; F.slopeOut = T.slopeOut; F.coefOut = T.coefOut; F.massOut = T.massOut;
    F.LofE = Spline1dView{ static_cast<int>(T.lofe.size() / 4), A->lofe.ptr };
    F.RofL = Spline1dView{ static_cast<int>(T.rofl.size() / 4), A->rofl.ptr };
    F.PhiofR = Spline1dView{ static_cast<int>(T.phiofr.size() / 4), A->phiofr.ptr };
    return A;
}

}  // namespace agb
