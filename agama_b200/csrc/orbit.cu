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
#include <map>
#include <mutex>

namespace agb {

namespace {

constexpr int ORBIT_BLOCK = 64;
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
    i integrates orbit i only. */
template<int KIND>
__global__ void __launch_bounds__(ORBIT_BLOCK) dop853Kernel(const __grid_constant__ MultipoleView M, const OrbitParams P,
    long n, const double* __restrict__ ic, const double* __restrict__ T, double* __restrict__ out,
    long* __restrict__ nsteps, long* __restrict__ nrej, int* __restrict__ status,
    unsigned long long* queue)
{
    using namespace dp853;
    extern __shared__ double smem[];
    __shared__ StageTable tab;
    for(int k = threadIdx.x; k < static_cast<int>(sizeof(StageTable) / sizeof(double)); k += blockDim.x)
        reinterpret_cast<double*>(&tab)[k] = reinterpret_cast<const double*>(&STAGE_TABLE)[k];
    __syncthreads();
    const StageStore S{ smem + threadIdx.x, static_cast<int>(blockDim.x) };
    const double Om = P.Omega;

    long i = queue ? -1 : blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if(!queue && i >= n) return;
    int phase = queue ? PH_FETCH : PH_INIT1;
    double x[6], k1[6], xt[6], k1b[6];
    double t = 0, tEnd = 0, sign = 1, h = 0, h1 = 0, hNext = 0, accFac = 1, preverr = INFINITY, tb = 0, hLast = 0,
        remaining = 0;
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
            i = static_cast<long>(atomicAdd(queue, 1ull));
            if(i >= n) break;
            phase = PH_INIT1;
        }
        if(phase == PH_INIT1) {          // a new orbit: load its start
            for(int c = 0; c < 6; c++) x[c] = ic[6 * i + c];
            tEnd = T[i];
            t = 0; tb = 0; hLast = 0; steps = 0; rejects = 0; st = ORBIT_OK; accFac = 1;
            sign = tEnd >= 0 ? 1 : -1;
        }
        if(phase == PH_FINISH) {
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
        orbitRHS<3, KIND>(M, Om, tt, xt, k, wantAcc ? &af : nullptr);
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

void launchOrbits(const MultipoleView& M, const OrbitParams& P, long n, const double* ic, const double* T,
    double* out, long* nsteps, long* nrej, int* status, unsigned long long* queue, cudaStream_t stream)
{
    if(n <= 0) return;
    const int block = ORBIT_BLOCK;
    const size_t shmem = orbitSharedBytes(block);
    const int kind = evalKindOf(M);
    auto kernel = kind == EVAL_AXI ? dop853Kernel<EVAL_AXI> : kind == EVAL_FAST ? dop853Kernel<EVAL_FAST>
                                                                              : dop853Kernel<EVAL_GENERAL>;
    long grid;
    if(queue) {
        int dev, sms, perSM = 0;
        AGB_CUDA(cudaGetDevice(&dev));
        AGB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        AGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, block, shmem));
        grid = static_cast<long>(sms) * (perSM > 0 ? perSM : 1);
        const long needed = (n + block - 1) / block;
        if(grid > needed) grid = needed;
        AGB_CUDA(cudaMemsetAsync(queue, 0, sizeof(unsigned long long), stream));
    } else {
        grid = (n + block - 1) / block;
    }
    kernel<<<grid, block, shmem, stream>>>(M, P, n, ic, T, out, nsteps, nrej, status, queue);
    AGB_CUDA(cudaGetLastError());
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
    // launchOrbits clears the counter (cudaMemsetAsync on the stream) before the kernel runs
    launchOrbits(M, P, n, ic, T, out, nsteps, nrej, status, base + slot, stream);
}

}  // namespace agb
