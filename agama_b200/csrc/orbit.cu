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

/// integrate one orbit; writes the final point (rotating frame), counters and status
template<int KIND>
__device__ void integrateOrbit(const MultipoleView& M, const OrbitParams& P, const double* ic,
    double tEnd, const StageStore& S, double* out, long* nAccepted, long* nRejected, int* status)
{
    using namespace dp853;
    const double Om = P.Omega;
    double x[6], k1[6], xt[6], k13[6];
    for(int c = 0; c < 6; c++) x[c] = ic[c];
    double t = 0;
    long steps = 0, rejects = 0;
    int st = ORBIT_OK;
    // --- init: derivatives at the start and the initial step (OdeStepperDOP853::init)
    double accFac = 1;
    orbitRHS<3, KIND>(M, Om, t, x, k1, &accFac);
    double hNext;
    {
        // initTimeStep (src/math_ode.cpp:35-91): Euler + Heun probes, Aarseth-like estimate
        double nx = 0, nd = 0;
        for(int c = 0; c < 6; c++) { nx += x[c] * x[c]; nd += k1[c] * k1[c]; }
        const double h1 = fmax(HMIN, fmin(HMAX, sqrt(nx / nd) * 0.01));
        double k2[6], k3[6];
        for(int c = 0; c < 6; c++) xt[c] = x[c] + h1 * k1[c];
        orbitRHS<3, KIND>(M, Om, t + h1, xt, k2, nullptr);
        for(int c = 0; c < 6; c++) xt[c] = x[c] + 0.5 * h1 * (k1[c] + k2[c]);
        orbitRHS<3, KIND>(M, Om, t + h1, xt, k3, nullptr);
        double h2 = INFINITY;
        for(int c = 0; c < 6; c++) {
            const double d0 = fmax(P.accAbs, fmax(fabs(x[c]), fabs(xt[c])));
            const double d1 = fmax(fabs(k1[c]), fabs(k3[c]));
            const double d2 = fabs((3 * k2[c] - k1[c] - 2 * k3[c]) / h1);
            const double d3 = fabs(6 * (k3[c] - k2[c]) / (h1 * h1));
            h2 = fmin(h2, (d0 * d2 + d1 * d1) / (d1 * d3 + d2 * d2));
        }
        hNext = fmax(HMIN, fmin(HMAX, pow(P.accRel, 1. / 8) * sqrt(h2))) * accFac;
    }
    double tb = 0, hLast = 0;
    if(tEnd != 0 && isFinite(tEnd)) {
        const double sign = tEnd >= 0 ? 1 : -1;
        while(t != tEnd) {
            const double remaining = tEnd - t;
            double h = fmin(remaining * sign, hNext) * sign;
            int nbad = 0, attempts = 0;
            double preverr = INFINITY;
            bool accepted = false;
            while(!accepted) {
                if(h == 0 || !isFinite(h) || ++attempts > MAX_ATTEMPTS_PER_STEP) { st = ORBIT_BAD_STEP; break; }
                // ---- the twelve stages (xt = x + h * sum a_ij k_j), then k13 at the end point
                for(int c = 0; c < 6; c++) xt[c] = x[c] + h * a21 * k1[c];
                { double k[6]; orbitRHS<3, KIND>(M, Om, t + c2 * h, xt, k, nullptr); for(int c = 0; c < 6; c++) S.at(0, c) = k[c]; }
                for(int c = 0; c < 6; c++) xt[c] = x[c] + h * (a31 * k1[c] + a32 * S.at(0, c));
                { double k[6]; orbitRHS<3, KIND>(M, Om, t + c3 * h, xt, k, nullptr); for(int c = 0; c < 6; c++) S.at(1, c) = k[c]; }
                for(int c = 0; c < 6; c++) xt[c] = x[c] + h * (a41 * k1[c] + a43 * S.at(1, c));
                { double k[6]; orbitRHS<3, KIND>(M, Om, t + c4 * h, xt, k, nullptr); for(int c = 0; c < 6; c++) S.at(2, c) = k[c]; }
                for(int c = 0; c < 6; c++) xt[c] = x[c] + h * (a51 * k1[c] + a53 * S.at(1, c) + a54 * S.at(2, c));
                { double k[6]; orbitRHS<3, KIND>(M, Om, t + c5 * h, xt, k, nullptr); for(int c = 0; c < 6; c++) S.at(3, c) = k[c]; }
                for(int c = 0; c < 6; c++) xt[c] = x[c] + h * (a61 * k1[c] + a64 * S.at(2, c) + a65 * S.at(3, c));
                { double k[6]; orbitRHS<3, KIND>(M, Om, t + c6 * h, xt, k, nullptr); for(int c = 0; c < 6; c++) S.at(4, c) = k[c]; }
                for(int c = 0; c < 6; c++)
                    xt[c] = x[c] + h * (a71 * k1[c] + a74 * S.at(2, c) + a75 * S.at(3, c) + a76 * S.at(4, c));
                { double k[6]; orbitRHS<3, KIND>(M, Om, t + c7 * h, xt, k, nullptr); for(int c = 0; c < 6; c++) S.at(5, c) = k[c]; }
                for(int c = 0; c < 6; c++)
                    xt[c] = x[c] + h * (a81 * k1[c] + a84 * S.at(2, c) + a85 * S.at(3, c) + a86 * S.at(4, c) +
                        a87 * S.at(5, c));
                { double k[6]; orbitRHS<3, KIND>(M, Om, t + c8 * h, xt, k, nullptr); for(int c = 0; c < 6; c++) S.at(6, c) = k[c]; }
                for(int c = 0; c < 6; c++)
                    xt[c] = x[c] + h * (a91 * k1[c] + a94 * S.at(2, c) + a95 * S.at(3, c) + a96 * S.at(4, c) +
                        a97 * S.at(5, c) + a98 * S.at(6, c));
                { double k[6]; orbitRHS<3, KIND>(M, Om, t + c9 * h, xt, k, nullptr); for(int c = 0; c < 6; c++) S.at(7, c) = k[c]; }
                for(int c = 0; c < 6; c++)
                    xt[c] = x[c] + h * (a101 * k1[c] + a104 * S.at(2, c) + a105 * S.at(3, c) + a106 * S.at(4, c) +
                        a107 * S.at(5, c) + a108 * S.at(6, c) + a109 * S.at(7, c));
                { double k[6]; orbitRHS<3, KIND>(M, Om, t + c10 * h, xt, k, nullptr); for(int c = 0; c < 6; c++) S.at(8, c) = k[c]; }
                // stage 11 -> slot of k2, stage 12 -> slot of k3
                for(int c = 0; c < 6; c++)
                    xt[c] = x[c] + h * (a111 * k1[c] + a114 * S.at(2, c) + a115 * S.at(3, c) + a116 * S.at(4, c) +
                        a117 * S.at(5, c) + a118 * S.at(6, c) + a119 * S.at(7, c) + a1110 * S.at(8, c));
                { double k[6]; orbitRHS<3, KIND>(M, Om, t + c11 * h, xt, k, nullptr); for(int c = 0; c < 6; c++) S.at(0, c) = k[c]; }
                for(int c = 0; c < 6; c++)
                    xt[c] = x[c] + h * (a121 * k1[c] + a124 * S.at(2, c) + a125 * S.at(3, c) + a126 * S.at(4, c) +
                        a127 * S.at(5, c) + a128 * S.at(6, c) + a129 * S.at(7, c) + a1210 * S.at(8, c) +
                        a1211 * S.at(0, c));
                { double k[6]; orbitRHS<3, KIND>(M, Om, t + h, xt, k, nullptr); for(int c = 0; c < 6; c++) S.at(1, c) = k[c]; }
                double k1b[6];
                for(int c = 0; c < 6; c++) {
                    k1b[c] = b1 * k1[c] + b6 * S.at(4, c) + b7 * S.at(5, c) + b8 * S.at(6, c) + b9 * S.at(7, c) +
                        b10 * S.at(8, c) + b11 * S.at(0, c) + b12 * S.at(1, c);
                    xt[c] = x[c] + h * k1b[c];
                }
                double af = 1;
                orbitRHS<3, KIND>(M, Om, t + h, xt, k13, &af);
                // ---- error estimate (3rd and 5th order embedded solutions)
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
                if(!isFinite(err)) { st = ORBIT_NONFINITE; break; }
                double fac = sqrt(sqrt(sqrt(err)));
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
                    }
                }
            }
            if(st != ORBIT_OK) break;
            for(int c = 0; c < 6; c++) { x[c] = xt[c]; k1[c] = k13[c]; }
            tb = t;
            hLast = h;
            t = h == remaining ? tEnd : t + h;
            if(++steps >= P.maxSteps) { if(t != tEnd) st = ORBIT_MAX_STEPS; break; }
        }
    }
    // final point in the rotating frame at time tb + hLast (RuntimeTrajectory semantics)
    double ca = 1, sa = 0;
    if(Om != 0) sincos(Om * (hLast + tb), &sa, &ca);
    out[0] = x[0] * ca + x[1] * sa;
    out[1] = x[1] * ca - x[0] * sa;
    out[2] = x[2];
    out[3] = x[3] * ca + x[4] * sa;
    out[4] = x[4] * ca - x[3] * sa;
    out[5] = x[5];
    *nAccepted = steps;
    *nRejected = rejects;
    *status = st;
}

/// one orbit per thread (queue == nullptr) or a persistent grid draining a work queue
template<int KIND>
__global__ void __launch_bounds__(ORBIT_BLOCK) dop853Kernel(const __grid_constant__ MultipoleView M, const OrbitParams P,
    long n, const double* __restrict__ ic, const double* __restrict__ T, double* __restrict__ out,
    long* __restrict__ nsteps, long* __restrict__ nrej, int* __restrict__ status,
    unsigned long long* queue)
{
    extern __shared__ double smem[];
    const StageStore S{ smem + threadIdx.x, static_cast<int>(blockDim.x) };
    long i = queue ? static_cast<long>(atomicAdd(queue, 1ull)) : blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    while(i < n) {
        double o[6];
        long na, nr;
        int s;
        integrateOrbit<KIND>(M, P, ic + 6 * i, T[i], S, o, &na, &nr, &s);
        for(int c = 0; c < 6; c++) out[6 * i + c] = o[c];
        if(nsteps) nsteps[i] = na;
        if(nrej) nrej[i] = nr;
        if(status) status[i] = s;
        if(!queue) break;
        i = static_cast<long>(atomicAdd(queue, 1ull));
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
