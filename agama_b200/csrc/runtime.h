// Host runtime shared by the C-ABI entry points: error reporting, CUDA checks and the
// device-resident objects behind the opaque handles.
#pragma once
#include <string>
#include <stdexcept>
#include <vector>
#include <cuda_runtime.h>
#include "multipole.h"
#include "fudge_types.h"

namespace agb {

/// last error message of the calling thread (the reference keeps one global string,
/// src/interface_c.cpp:5-7; a per-thread string keeps concurrent callers apart)
void setError(const std::string& msg);
const char* lastError();

#define AGB_CUDA(call) do { cudaError_t e_ = (call); if(e_ != cudaSuccess) \
    throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #call); } while(0)

/// throws if no CUDA device is usable: the engine has no CPU fallback
void requireDevice();

/// device buffer (RAII)
template<typename T>
struct DevBuf {
    T* ptr = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { if(ptr) cudaFree(ptr); }
    void alloc(size_t count) {
        if(ptr) { cudaFree(ptr); ptr = nullptr; }
        n = count;
        if(count) AGB_CUDA(cudaMalloc(&ptr, count * sizeof(T)));
    }
    void upload(const std::vector<T>& v) {
        alloc(v.size());
        if(!v.empty()) AGB_CUDA(cudaMemcpy(ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    }
};

/// a Multipole potential resident on one device
struct DevicePotential {
    int device = 0;
    MultipoleHost host;
    DevBuf<double> lnr, tau, lnrInvH, tauInvH, spl2d, spl1d, innerS, innerU, innerW, outerS, outerU, outerW;
    DevBuf<float> spl2d32;
    MultipoleView view;
    /// the axisymmetric (m = 0) part, used by the action finder (same as the full potential
    /// when the potential is axisymmetric)
    bool axisymmetric = false;
};

DevicePotential* createDevicePotential(const std::vector<double>& radii,
    const std::vector<std::vector<double>>& Phi, const std::vector<std::vector<double>>& dPhi);

struct OrbitParams;

struct Mlp;

/// a Staeckel-fudge action finder: tables on the device of its potential
struct DeviceActionFinder {
    DevicePotential* pot = nullptr;   // not owned
    FinderTablesHost host;
    DevBuf<double> gridE, gridL, delta, lofe, rofl, phiofr;
    FudgeTables view;
    Mlp* brackets = nullptr;          // owned; null until a predictor is trained
    float bracketWidths[3] = { 0, 0, 0 };
    bool useBrackets = false;
    bool countBrackets = true;        // the search counters are kept (bracketStats)
    DevBuf<unsigned long long> bracketStats;
    ~DeviceActionFinder();
};
DeviceActionFinder* createDeviceActionFinder(DevicePotential* pot, const FinderTablesHost& T);
/// build the focal-distance table and the L_circ interpolator of a potential (finder_build.cu)
FinderTablesHost buildFinderTables(const DevicePotential& P);

/// launch helpers (defined in the .cu files)
/// (cylindrical: points (R, z, phi) and derivatives in cylindrical coordinates)
void launchEvalPotential(const MultipoleView& M, long n, const double* pos, double* phi,
    double* grad, double* hess, cudaStream_t stream, bool cylindrical = false);
/// density (Laplacian / 4 pi inside the grid, closed form outside) at n Cartesian points
void launchDensity(const MultipoleView& M, long n, const double* pos, double* rho, cudaStream_t stream);
/// radius queries in the equatorial plane of the azimuthally averaged potential: a = E (or L for
/// RADIUS_CIRC_L), b = L (RADIUS_PERIAPO only); out1 = radius (pericentre), out2 = apocentre
enum RadiusQuery { RADIUS_CIRC_E = 0, RADIUS_CIRC_L = 1, RADIUS_MAX = 2, RADIUS_PERIAPO = 3 };
void launchRadii(const MultipoleView& M, int query, long n, const double* a, const double* b, double* out1,
    double* out2, cudaStream_t stream);
/// launch shape of an orbit batch: lanes of a warp per orbit (1, 2, 4, 8) and threads per block
/// (32, 64, 128); 0 = chosen by the autotuner.  Neither changes any result bit.
struct OrbitShape { int lanes = 0, block = 0; };
/// DOP853 batch; queue != nullptr selects the persistent work-queue mapping (8-byte counter)
void launchOrbits(const MultipoleView& M, const OrbitParams& P, long n, const double* ic, const double* T,
    double* out, long* nsteps, long* nrej, int* status, unsigned long long* queue, cudaStream_t stream,
    OrbitShape shape = OrbitShape());
/// phase timing of the action computation: on = true clears and starts recording; on = false
/// stops and returns the summed device durations (ms) of prepare, bracket inference, root
/// searches and integrals, and the number of passes timed
void setActionPhaseTiming(bool on, double* ms, long* passes);
/// mixed precision for the action integrals of later calls: the integrand's arithmetic after
/// F(tau) and the Gauss-Legendre sums in FP32 (compensated); false (default) = all FP64
void setActionMixedPrecision(bool mixed);
/// lanes per orbit for all later batches: 1, 2, 4, 8, or 0 (default) for the autotuner
void setOrbitLanes(int lanes);
/// threads per block of the orbit kernels for all later batches: 32, 64, 128, or 0 (default)
/// for the autotuner
void setOrbitBlock(int block);
/// mixed precision for later batches in multi-harmonic potentials: the m != 0 harmonics of the
/// force from an FP32 copy of the spline table (one lane per orbit); false (default) = all FP64
void setOrbitMixedPrecision(bool mixed);
/// the launch shape a batch will use (runs the autotuner's trial on the stream if needed)
OrbitShape orbitShapeFor(const MultipoleView& M, const OrbitParams& P, long n, const double* ic, const double* T,
    cudaStream_t stream);

/// the same work-queue batch with its counter in the library's static device array (slot 0..31),
/// allocating nothing
void launchOrbitsNoAlloc(const MultipoleView& M, const OrbitParams& P, long n, const double* ic, const double* T,
    double* out, long* nsteps, long* nrej, int* status, int slot, cudaStream_t stream);
int noallocQueueSlots();
/// Staeckel fudge with a given focal distance per point (fd) or one for all (fd0 when fd is null);
/// outputs n x 3 each: actions (Jr, Jz, Jphi), angles and frequencies (any of them may be null)
void launchActionsFixedDelta(const MultipoleView& M, long n, const double* posvel, const double* fd, double fd0,
    double* act, double* ang, double* freq, int* iters, cudaStream_t stream);
/// a trained bracket predictor attached to an action finder: the network, the half-widths of its
/// brackets (nu_max, lambda_min, lambda_max; see fudgeRootKernel) and 4 device counters
/// {searches, narrowed, fallbacks, iterations} (may be null)
struct BracketPlan { const Mlp* net; float widths[3]; unsigned long long* stats; };
/// outputs of launchBracketSamples (device arrays n x 6, n x 3, n x 3)
struct BracketSamples { float* features; float* target; float* mask; };

/// Staeckel fudge with the focal distance from the action finder's table (bp: optional predictor)
void launchActionsFinder(const MultipoleView& M, const FudgeTables& F, long n, const double* posvel,
    double* act, double* ang, double* freq, double* fdOut, int* iters, cudaStream_t stream,
    const BracketPlan* bp = nullptr);
/// the predictor's inputs and training targets of n points (plain root searches)
void launchBracketSamples(const MultipoleView& M, const FudgeTables& F, long n, const double* posvel,
    const BracketSamples& samples, cudaStream_t stream);

}  // namespace agb
