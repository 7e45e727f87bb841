// C-ABI of the B200 engine: the entry points of the reference's plain-C interface
// (src/interface_c.h) for the Multipole / orbit / Staeckel-fudge path, plus batched and
// device-pointer variants.  No exception crosses this boundary: constructors return NULL and
// batched calls return a non-zero status, with the message in agama_getError().
#include "runtime.h"
#include "host_pipeline.h"
#include "mlp.h"
#include "../../include/agama_b200.h"
#include <cstring>
#include <algorithm>
#include <cmath>
#include <sstream>
#include <cctype>
#include <map>

using namespace agb;

struct agama_Potential { DevicePotential* pot; };

namespace {

std::string trimStr(const std::string& s) {
    size_t a = s.find_first_not_of(" \t"), b = s.find_last_not_of(" \t");
    return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}
std::string lowerStr(std::string s) { for(auto& c : s) c = static_cast<char>(tolower(c)); return s; }

/// key=value pairs of a parameter string ("key=value, key=value" or separated by newlines /
/// semicolons), keys in lower case (the reference's KeyValueMap, case-insensitive keys)
std::map<std::string, std::string> parseKeyValues(const char* params)
{
    std::map<std::string, std::string> kv;
    std::string text = params ? params : "";
    for(auto& c : text) if(c == ';' || c == '\n') c = ',';
    std::stringstream ss(text);
    std::string item;
    while(std::getline(ss, item, ',')) {
        const size_t eq = item.find('=');
        if(eq == std::string::npos) continue;
        kv[lowerStr(trimStr(item.substr(0, eq)))] = trimStr(item.substr(eq + 1));
    }
    return kv;
}

/// the Multipole's own parameters; every other key describes the density
const char* const MULTIPOLE_KEYS[] = { "type", "lmax", "mmax", "gridsizer", "rmin", "rmax", "symmetry", "fixorder",
    "density", "file" };

bool isMultipoleKey(const std::string& k)
{
    for(const char* m : MULTIPOLE_KEYS) if(k == m) return true;
    return false;
}

/** a potential from the reference's key=value parameters (createPotential for a single section,
    src/potential_factory.cpp:1376-1441, as the plain-C agama_createPotential passes them,
    src/interface_c.cpp:31-51): "file=<Multipole coefficient file>" (type=Multipole optional),
    or "type=Multipole, density=<Dehnen|Plummer|NFW|MiyamotoNagai|Spheroid|Disk>, <density
    parameters>, lmax, mmax, gridSizeR, rmin, rmax, symmetry" (the Poisson solve) */
DevicePotential* potentialFromParams(const char* params)
{
    if(!params) throw std::invalid_argument("createPotential: null parameter string");
    const std::map<std::string, std::string> kv = parseKeyValues(params);
    auto typeIt = kv.find("type");
    const std::string type = typeIt == kv.end() ? "" : lowerStr(typeIt->second);
    if(!type.empty() && type != "multipole")
        throw std::invalid_argument("createPotential: only type=Multipole is supported (from a coefficient file or "
            "a density model)");
    std::vector<double> radii;
    std::vector<std::vector<double>> Phi, dPhi;
    if(kv.count("file")) {
        for(const auto& e : kv)
            if(e.first != "file" && e.first != "type")
                throw std::invalid_argument("createPotential: parameter '" + e.first + "' is not used with file=");
        readMultipoleCoefFile(kv.at("file"), radii, Phi, dPhi);
    } else if(kv.count("density")) {
        std::map<std::string, std::string> dens, mp;
        for(const auto& e : kv) {
            if(e.first == "density") dens["type"] = e.second;
            else if(isMultipoleKey(e.first)) mp[e.first] = e.second;
            else dens[e.first] = e.second;
        }
        multipoleCoefsFromDensity({ dens }, mp, radii, Phi, dPhi);
    } else
        throw std::invalid_argument("createPotential: give a coefficient file (file=...) or a density model "
            "(density=...)");
    return createDevicePotential(radii, Phi, dPhi);
}

/// restores the caller's current device when an entry point returns (the entry points make the
/// device of their object current for their own work)
struct CurrentDeviceGuard {
    int device = -1;
    CurrentDeviceGuard() { if(cudaGetDevice(&device) != cudaSuccess) { device = -1; cudaGetLastError(); } }
    ~CurrentDeviceGuard() { if(device >= 0) cudaSetDevice(device); }
    CurrentDeviceGuard(const CurrentDeviceGuard&) = delete;
    CurrentDeviceGuard& operator=(const CurrentDeviceGuard&) = delete;
};

template<class F>
int guarded(F&& f) {
    CurrentDeviceGuard keep;
    try { f(); return 0; }
    catch(std::exception& e) { setError(e.what()); return -1; }
}

}  // namespace

extern "C" {

const char* agama_getError() { return lastError(); }

agama_Potential* agama_createPotential(const char* params)
{
    try {
        return new agama_Potential{ potentialFromParams(params) };
    } catch(std::exception& e) {
        setError(e.what());
        return nullptr;
    }
}

agama_Potential* agama_createMultipoleFromDensities(const char* multipoleParams, int numComponents,
    const char* const* densityParams)
{
    try {
        if(numComponents < 1 || !densityParams) throw std::invalid_argument("createMultipoleFromDensities: no density");
        std::vector<double> radii;
        std::vector<std::vector<double>> Phi, dPhi;
        std::vector<std::map<std::string, std::string>> dens;
        for(int k = 0; k < numComponents; k++) dens.push_back(parseKeyValues(densityParams[k]));
        multipoleCoefsFromDensity(dens, parseKeyValues(multipoleParams), radii, Phi, dPhi);
        return new agama_Potential{ createDevicePotential(radii, Phi, dPhi) };
    } catch(std::exception& e) {
        setError(e.what());
        return nullptr;
    }
}

int agama_multipoleCoefsFromDensities(const char* multipoleParams, int numComponents,
    const char* const* densityParams, int* gridSizeR, int* numCoefs, double* radii, double* Phi, double* dPhi)
{
    // host-only: the Poisson solve without a device; call with radii == NULL to get the sizes
    return guarded([&] {
        if(numComponents < 1 || !densityParams || !gridSizeR || !numCoefs)
            throw std::invalid_argument("multipoleCoefsFromDensities: invalid arguments");
        std::vector<double> r;
        std::vector<std::vector<double>> P, D;
        std::vector<std::map<std::string, std::string>> dens;
        for(int k = 0; k < numComponents; k++) dens.push_back(parseKeyValues(densityParams[k]));
        multipoleCoefsFromDensity(dens, parseKeyValues(multipoleParams), r, P, D);
        const int nr = static_cast<int>(r.size()), nc = static_cast<int>(P.size());
        if(radii) {
            if(*gridSizeR < nr || *numCoefs < nc || !Phi || !dPhi)
                throw std::invalid_argument("multipoleCoefsFromDensities: output arrays too small");
            std::copy(r.begin(), r.end(), radii);
            for(int c = 0; c < nc; c++) {
                std::copy(P[c].begin(), P[c].end(), Phi + static_cast<size_t>(c) * nr);
                std::copy(D[c].begin(), D[c].end(), dPhi + static_cast<size_t>(c) * nr);
            }
        }
        *gridSizeR = nr;
        *numCoefs = nc;
    });
}

agama_Potential* agama_createMultipoleFromCoefs(int gridSizeR, const double* radii, int numCoefs,
    const double* Phi, const double* dPhi)
{
    try {
        if(gridSizeR < 2 || numCoefs < 1 || !radii || !Phi || !dPhi)
            throw std::invalid_argument("createMultipoleFromCoefs: invalid arguments");
        std::vector<double> r(radii, radii + gridSizeR);
        std::vector<std::vector<double>> P(numCoefs), D(numCoefs);
        for(int c = 0; c < numCoefs; c++) {
            P[c].assign(Phi + static_cast<size_t>(c) * gridSizeR, Phi + static_cast<size_t>(c + 1) * gridSizeR);
            D[c].assign(dPhi + static_cast<size_t>(c) * gridSizeR, dPhi + static_cast<size_t>(c + 1) * gridSizeR);
        }
        return new agama_Potential{ createDevicePotential(r, P, D) };
    } catch(std::exception& e) {
        setError(e.what());
        return nullptr;
    }
}

void agama_deletePotential(agama_Potential* p)
{
    if(!p) return;
    delete p->pot;
    delete p;
}

int agama_getPotentialInfo(const agama_Potential* p, int* lmax, int* mmax, int* symmetry,
    int* gridSizeR, int* gridSizeTau)
{
    return guarded([&] {
        if(!p) throw std::invalid_argument("null potential");
        const MultipoleHost& H = p->pot->host;
        if(lmax) *lmax = H.ind.lmax;
        if(mmax) *mmax = H.ind.mmax;
        if(symmetry) *symmetry = H.ind.sym;
        if(gridSizeR) *gridSizeR = static_cast<int>(H.radii.size());
        if(gridSizeTau) *gridSizeTau = static_cast<int>(H.tau.size());
    });
}

int agama_evalPotentialManyDevice(const agama_Potential* p, long n, const double* pos,
    double* phi, double* deriv, double* deriv2, void* stream)
{
    return guarded([&] {
        if(!p || n < 0 || (n > 0 && !pos)) throw std::invalid_argument("evalPotentialManyDevice: invalid arguments");
        AGB_CUDA(cudaSetDevice(p->pot->device));
        launchEvalPotential(p->pot->view, n, pos, phi, deriv, deriv2, static_cast<cudaStream_t>(stream));
    });
}

int agama_evalPotentialMany(const agama_Potential* p, long n, const double* pos, double time,
    double* phi, double* deriv, double* deriv2)
{
    (void)time;   // the Multipole potential is static
    return guarded([&] {
        if(!p || n < 0 || (n > 0 && !pos)) throw std::invalid_argument("evalPotentialMany: invalid arguments");
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(p->pot->device));
        const MultipoleView& M = p->pot->view;
        runChunked(n, { { pos, 3 * sizeof(double) } },
            { { phi, sizeof(double) }, { deriv, 3 * sizeof(double) }, { deriv2, 6 * sizeof(double) } },
            [&](long, long count, void* const* in, void* const* out, cudaStream_t s) {
                launchEvalPotential(M, count, static_cast<const double*>(in[0]), static_cast<double*>(out[0]),
                    static_cast<double*>(out[1]), static_cast<double*>(out[2]), s);
            });
    });
}

int agama_evalPotentialCylManyDevice(const agama_Potential* p, long n, const double* pos,
    double* phi, double* deriv, double* deriv2, void* stream)
{
    return guarded([&] {
        if(!p || n < 0 || (n > 0 && !pos)) throw std::invalid_argument("evalPotentialCylManyDevice: invalid arguments");
        AGB_CUDA(cudaSetDevice(p->pot->device));
        launchEvalPotential(p->pot->view, n, pos, phi, deriv, deriv2, static_cast<cudaStream_t>(stream), true);
    });
}

int agama_evalPotentialCylMany(const agama_Potential* p, long n, const double* pos, double time,
    double* phi, double* deriv, double* deriv2)
{
    (void)time;
    return guarded([&] {
        if(!p || n < 0 || (n > 0 && !pos)) throw std::invalid_argument("evalPotentialCylMany: invalid arguments");
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(p->pot->device));
        const MultipoleView& M = p->pot->view;
        runChunked(n, { { pos, 3 * sizeof(double) } },
            { { phi, sizeof(double) }, { deriv, 3 * sizeof(double) }, { deriv2, 6 * sizeof(double) } },
            [&](long, long count, void* const* in, void* const* out, cudaStream_t s) {
                launchEvalPotential(M, count, static_cast<const double*>(in[0]), static_cast<double*>(out[0]),
                    static_cast<double*>(out[1]), static_cast<double*>(out[2]), s, true);
            });
    });
}

double agama_evalPotential(const agama_Potential* p, const double pos[3], double time,
    double deriv[3], double deriv2[6])
{
    double phi = NAN;
    if(agama_evalPotentialMany(p, 1, pos, time, &phi, deriv, deriv2) != 0)
        return NAN;
    return phi;
}

// ---- density of a potential

agama_Density* agama_createDensity(const char* params)
{
    (void)params;
    setError("createDensity: density models are not part of the B200 engine; a potential created by "
             "agama_createPotential can be passed to agama_evalDensity instead");
    return nullptr;
}

void agama_deleteDensity(agama_Density* density) { (void)density; }

int agama_evalDensityManyDevice(const agama_Potential* p, long n, const double* pos, double* rho, void* stream)
{
    return guarded([&] {
        if(!p || n < 0 || (n > 0 && (!pos || !rho))) throw std::invalid_argument("evalDensityManyDevice: invalid arguments");
        AGB_CUDA(cudaSetDevice(p->pot->device));
        launchDensity(p->pot->view, n, pos, rho, static_cast<cudaStream_t>(stream));
    });
}

int agama_evalDensityMany(const agama_Potential* p, long n, const double* pos, double time, double* rho)
{
    (void)time;
    return guarded([&] {
        if(!p || n < 0 || (n > 0 && (!pos || !rho))) throw std::invalid_argument("evalDensityMany: invalid arguments");
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(p->pot->device));
        const MultipoleView& M = p->pot->view;
        runChunked(n, { { pos, 3 * sizeof(double) } }, { { rho, sizeof(double) } },
            [&](long, long count, void* const* in, void* const* out, cudaStream_t s) {
                launchDensity(M, count, static_cast<const double*>(in[0]), static_cast<double*>(out[0]), s);
            });
    });
}

double agama_evalDensity(const agama_Density* density, const double pos[3], double time)
{
    // the only objects with a density here are potentials (agama_createDensity makes none)
    double rho = NAN;
    if(agama_evalDensityMany(reinterpret_cast<const agama_Potential*>(density), 1, pos, time, &rho) != 0)
        return NAN;
    return rho;
}

// ---- radii of circular, radial and planar orbits

int agama_potentialRadiiManyDevice(const agama_Potential* p, int query, long n, const double* in1,
    const double* in2, double* out1, double* out2, void* stream)
{
    return guarded([&] {
        if(!p || n < 0 || (n > 0 && (!in1 || !out1 || (query == RADIUS_PERIAPO && (!in2 || !out2)))))
            throw std::invalid_argument("potentialRadiiManyDevice: invalid arguments");
        AGB_CUDA(cudaSetDevice(p->pot->device));
        launchRadii(p->pot->view, query, n, in1, in2, out1, out2, static_cast<cudaStream_t>(stream));
    });
}

int agama_potentialRadiiMany(const agama_Potential* p, int query, long n, const double* in1, const double* in2,
    double* out1, double* out2)
{
    return guarded([&] {
        const bool two = query == RADIUS_PERIAPO;
        if(!p || n < 0 || (n > 0 && (!in1 || !out1 || (two && (!in2 || !out2)))))
            throw std::invalid_argument("potentialRadiiMany: invalid arguments");
        if(query < RADIUS_CIRC_E || query > RADIUS_PERIAPO)
            throw std::invalid_argument("potentialRadiiMany: unknown query " + std::to_string(query));
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(p->pot->device));
        const MultipoleView& M = p->pot->view;
        runChunked(n, { { in1, sizeof(double) }, { two ? in2 : nullptr, sizeof(double) } },
            { { out1, sizeof(double) }, { two ? out2 : nullptr, sizeof(double) } },
            [&](long, long count, void* const* in, void* const* out, cudaStream_t s) {
                launchRadii(M, query, count, static_cast<const double*>(in[0]), static_cast<const double*>(in[1]),
                    static_cast<double*>(out[0]), static_cast<double*>(out[1]), s);
            });
    });
}

double agama_R_circ(const agama_Potential* p, double E)
{
    double R = NAN;
    if(agama_potentialRadiiMany(p, RADIUS_CIRC_E, 1, &E, nullptr, &R, nullptr) != 0) return NAN;
    return R;
}

double agama_R_from_Lz(const agama_Potential* p, double Lz)
{
    double R = NAN;
    if(agama_potentialRadiiMany(p, RADIUS_CIRC_L, 1, &Lz, nullptr, &R, nullptr) != 0) return NAN;
    return R;
}

double agama_R_max(const agama_Potential* p, double E)
{
    double R = NAN;
    if(agama_potentialRadiiMany(p, RADIUS_MAX, 1, &E, nullptr, &R, nullptr) != 0) return NAN;
    return R;
}

void agama_findPlanarOrbitExtent(const agama_Potential* p, double E, double L, double* Rperi, double* Rapo)
{
    double R1 = NAN, R2 = NAN;
    if(agama_potentialRadiiMany(p, RADIUS_PERIAPO, 1, &E, &L, &R1, &R2) != 0) R1 = R2 = NAN;
    if(Rperi) *Rperi = R1;
    if(Rapo) *Rapo = R2;
}

}  // extern "C"

extern "C" int agama_inspectMultipoleFile(const char* file, int* lmax, int* mmax, int* symmetry,
    int* gridSizeR, int* gridSizeTau)
{
    // host-only: parse the file and build the tables without touching a device
    return guarded([&] {
        std::vector<double> radii;
        std::vector<std::vector<double>> Phi, dPhi;
        readMultipoleCoefFile(file ? file : "", radii, Phi, dPhi);
        MultipoleHost H = buildMultipole(radii, Phi, dPhi);
        if(lmax) *lmax = H.ind.lmax;
        if(mmax) *mmax = H.ind.mmax;
        if(symmetry) *symmetry = H.ind.sym;
        if(gridSizeR) *gridSizeR = static_cast<int>(H.radii.size());
        if(gridSizeTau) *gridSizeTau = static_cast<int>(H.tau.size());
    });
}

extern "C" int agama_writePotential(const char* fileName, const agama_Potential* p)
{
    return guarded([&] {
        if(!fileName || !p) throw std::invalid_argument("writePotential: invalid arguments");
        const MultipoleHost& H = p->pot->host;
        writeMultipoleCoefFile(fileName, H.radii, H.Phi, H.dPhi, H.ind.sym);
    });
}

extern "C" int agama_writeMultipoleCoefs(const char* fileName, int gridSizeR, const double* radii, int numCoefs,
    const double* Phi, const double* dPhi)
{
    // host-only: the tables are built to validate the coefficients and find their symmetry
    return guarded([&] {
        if(!fileName || gridSizeR < 2 || numCoefs < 1 || !radii || !Phi || !dPhi)
            throw std::invalid_argument("writeMultipoleCoefs: invalid arguments");
        std::vector<double> r(radii, radii + gridSizeR);
        std::vector<std::vector<double>> P(numCoefs), D(numCoefs);
        for(int c = 0; c < numCoefs; c++) {
            P[c].assign(Phi + static_cast<size_t>(c) * gridSizeR, Phi + static_cast<size_t>(c + 1) * gridSizeR);
            D[c].assign(dPhi + static_cast<size_t>(c) * gridSizeR, dPhi + static_cast<size_t>(c + 1) * gridSizeR);
        }
        const MultipoleHost H = buildMultipole(r, P, D);
        writeMultipoleCoefFile(fileName, H.radii, H.Phi, H.dPhi, H.ind.sym);
    });
}

// ------------------------------------------------------------------------------------------
// orbits

#include "dop853.cuh"

namespace {
OrbitParams makeOrbitParams(double Omega, double accuracy, long maxNumSteps)
{
    if(!(accuracy > 0)) throw std::invalid_argument("integrateOrbits: accuracy must be positive");
    OrbitParams P;
    P.Omega = Omega;
    P.accRel = accuracy;
    P.accAbs = 0;
    P.maxSteps = maxNumSteps > 0 ? maxNumSteps : 100000000L;   // reference default 1e8, src/orbit.h:127
    return P;
}
}  // namespace

extern "C" int agama_setOrbitLanesPerOrbit(int lanes)
{
    return guarded([&] {
        if(!(lanes == 0 || lanes == 1 || lanes == 2 || lanes == 4 || lanes == 8))
            throw std::invalid_argument("setOrbitLanesPerOrbit: lanes must be 0 (autotuned), 1, 2, 4 or 8");
        setOrbitLanes(lanes);
    });
}

extern "C" int agama_setActionPrecision(int mixed)
{
    return guarded([&] {
        if(mixed != 0 && mixed != 1) throw std::invalid_argument("setActionPrecision: 0 (FP64) or 1 (mixed)");
        setActionMixedPrecision(mixed == 1);
    });
}

extern "C" int agama_setOrbitBlockSize(int block)
{
    return guarded([&] {
        if(!(block == 0 || block == 32 || block == 64 || block == 128))
            throw std::invalid_argument("setOrbitBlockSize: block must be 0 (autotuned), 32, 64 or 128");
        setOrbitBlock(block);
    });
}

extern "C" int agama_setOrbitPrecision(int mixed)
{
    return guarded([&] {
        if(mixed != 0 && mixed != 1) throw std::invalid_argument("setOrbitPrecision: mixed must be 0 or 1");
        setOrbitMixedPrecision(mixed != 0);
    });
}

extern "C" int agama_integrateOrbitsManyDevice(const agama_Potential* p, long n, const double* ic,
    const double* T, double Omega, double accuracy, long maxNumSteps, double* finalState,
    long* numSteps, long* numRejected, int* status, int useQueue, void* stream)
{
    return guarded([&] {
        if(!p || n < 0 || (n > 0 && (!ic || !T || !finalState)))
            throw std::invalid_argument("integrateOrbitsManyDevice: invalid arguments");
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(p->pot->device));
        const OrbitParams P = makeOrbitParams(Omega, accuracy, maxNumSteps);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        unsigned long long* queue = nullptr;
        if(useQueue) AGB_CUDA(cudaMallocAsync(&queue, sizeof(unsigned long long), s));
        launchOrbits(p->pot->view, P, n, ic, T, finalState, numSteps, numRejected, status, queue, s);
        if(queue) AGB_CUDA(cudaFreeAsync(queue, s));
    });
}

extern "C" int agama_integrateOrbitsTrajectoryManyDevice(const agama_Potential* p, long n, const double* ic,
    const double* T, double Omega, double accuracy, long maxNumSteps, int trajSize, double* traj,
    double* finalState, long* numSteps, int* status, void* stream)
{
    return guarded([&] {
        if(!p || n < 0 || trajSize < 2 || (n > 0 && (!ic || !T || !traj || !finalState)))
            throw std::invalid_argument("integrateOrbitsTrajectoryManyDevice: invalid arguments (trajSize >= 2)");
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(p->pot->device));
        OrbitParams P = makeOrbitParams(Omega, accuracy, maxNumSteps);
        P.trajSize = trajSize;
        P.traj = traj;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        Scratch q(sizeof(unsigned long long), s);
        launchOrbits(p->pot->view, P, n, ic, T, finalState, numSteps, nullptr, status,
            static_cast<unsigned long long*>(q.ptr), s);
    });
}

extern "C" int agama_integrateOrbitsTrajectoryMany(const agama_Potential* p, long n, const double* ic,
    const double* T, double Omega, double accuracy, long maxNumSteps, int trajSize, double* traj,
    double* finalState, long* numSteps, int* status)
{
    return guarded([&] {
        if(!p || n < 0 || trajSize < 2 || (n > 0 && (!ic || !T || !traj)))
            throw std::invalid_argument("integrateOrbitsTrajectoryMany: invalid arguments (trajSize >= 2)");
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(p->pot->device));
        DevBuf<double> dic(6 * n), dT(n), dout(6 * n), dtraj(static_cast<size_t>(n) * trajSize * 6);
        DevBuf<long> dsteps(n);
        DevBuf<int> dstat(n);
        AGB_CUDA(cudaMemcpy(dic.ptr, ic, 6 * n * sizeof(double), cudaMemcpyHostToDevice));
        AGB_CUDA(cudaMemcpy(dT.ptr, T, n * sizeof(double), cudaMemcpyHostToDevice));
        if(agama_integrateOrbitsTrajectoryManyDevice(p, n, dic.ptr, dT.ptr, Omega, accuracy, maxNumSteps, trajSize,
                dtraj.ptr, dout.ptr, dsteps.ptr, dstat.ptr, nullptr) != 0)
            throw std::runtime_error(lastError());
        AGB_CUDA(cudaMemcpy(traj, dtraj.ptr, static_cast<size_t>(n) * trajSize * 6 * sizeof(double),
            cudaMemcpyDeviceToHost));
        if(finalState) AGB_CUDA(cudaMemcpy(finalState, dout.ptr, 6 * n * sizeof(double), cudaMemcpyDeviceToHost));
        if(numSteps) AGB_CUDA(cudaMemcpy(numSteps, dsteps.ptr, n * sizeof(long), cudaMemcpyDeviceToHost));
        if(status) AGB_CUDA(cudaMemcpy(status, dstat.ptr, n * sizeof(int), cudaMemcpyDeviceToHost));
    });
}

// ---- orbits with a target (runtime function accumulating a density grid)

struct agama_Target {
    int degree = 0, strips = 0;
    std::vector<double> shellRadii;
    double axisX = 1, axisY = 1, axisZ = 1;
    int valuesPerShell = 0, numValues = 0;
};

extern "C" agama_Target* agama_createTargetDensityClassic(int degree, int stripsPerPane, int gridSize,
    const double* gridr, double axisRatioY, double axisRatioZ)
{
    try {
        if(degree != 0 && degree != 1) throw std::invalid_argument("createTargetDensityClassic: degree must be 0 or 1");
        if(gridSize < 1 || !gridr) throw std::invalid_argument("createTargetDensityClassic: no radial grid");
        agama_Target* T = new agama_Target;
        T->degree = degree;
        T->strips = stripsPerPane;
        // TargetDensityClassic constructor (src/galaxymodel_densitygrid.cpp:149-167): a leading
        // zero node is implied and dropped; the axes keep the volume (axisX axisY axisZ = 1)
        const int first = gridr[0] > 0 ? 0 : 1;
        T->shellRadii.assign(gridr + first, gridr + gridSize);
        T->axisX = 1. / cbrt(axisRatioY * axisRatioZ);
        T->axisY = axisRatioY * T->axisX;
        T->axisZ = axisRatioZ * T->axisX;
        bool ok = T->shellRadii.size() >= 1 && T->shellRadii[0] > 0;
        for(size_t k = 1; k < T->shellRadii.size(); k++) ok &= T->shellRadii[k] > T->shellRadii[k - 1];
        if(!ok || stripsPerPane < 1 || !(axisRatioY > 0) || !(axisRatioZ > 0)) {
            delete T;
            throw std::invalid_argument("TargetDensityClassic: invalid grid parameters");
        }
        T->valuesPerShell = 3 * stripsPerPane * (stripsPerPane + degree) + degree;
        T->numValues = T->valuesPerShell * static_cast<int>(T->shellRadii.size()) + degree;
        return T;
    } catch(std::exception& e) {
        setError(e.what());
        return nullptr;
    }
}

extern "C" void agama_deleteTarget(agama_Target* target) { delete target; }

extern "C" int agama_targetNumCoefs(const agama_Target* target) { return target ? target->numValues : 0; }

extern "C" int agama_integrateOrbitsTargetManyDevice(const agama_Potential* p, long n, const double* ic,
    const double* T, double Omega, double accuracy, long maxNumSteps, const agama_Target* target, float* output,
    double* finalState, long* numSteps, int* status, void* stream)
{
    return guarded([&] {
        if(!p || !target || n < 0 || (n > 0 && (!ic || !T || !output || !finalState)))
            throw std::invalid_argument("integrateOrbitsTargetManyDevice: invalid arguments");
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(p->pot->device));
        OrbitParams P = makeOrbitParams(Omega, accuracy, maxNumSteps);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const size_t cubeBytes = static_cast<size_t>(n) * target->numValues * sizeof(double);
        const size_t radiiBytes = target->shellRadii.size() * sizeof(double);
        Scratch scratch(cubeBytes + radiiBytes + 512, s);
        double* cube = static_cast<double*>(scratch.ptr);
        double* radii = reinterpret_cast<double*>(static_cast<char*>(scratch.ptr) + cubeBytes);
        unsigned long long* queue = reinterpret_cast<unsigned long long*>(
            static_cast<char*>(scratch.ptr) + cubeBytes + ((radiiBytes + 255) / 256) * 256);
        AGB_CUDA(cudaMemsetAsync(cube, 0, cubeBytes, s));
        AGB_CUDA(cudaMemcpyAsync(radii, target->shellRadii.data(), radiiBytes, cudaMemcpyHostToDevice, s));
        TargetView& V = P.target;
        V.degree = target->degree;
        V.strips = target->strips;
        V.nShells = static_cast<int>(target->shellRadii.size());
        V.valuesPerShell = target->valuesPerShell;
        V.numValues = target->numValues;
        V.shellRadii = radii;
        V.axisX = target->axisX; V.axisY = target->axisY; V.axisZ = target->axisZ;
        V.datacube = cube;
        V.output = output;
        launchOrbits(p->pot->view, P, n, ic, T, finalState, numSteps, nullptr, status, queue, s);
        // the scratch (accumulators, radii) is released in stream order after the kernel
    });
}

extern "C" int agama_integrateOrbitsTargetMany(const agama_Potential* p, long n, const double* ic,
    const double* T, double Omega, double accuracy, long maxNumSteps, const agama_Target* target, float* output,
    double* finalState, long* numSteps, int* status)
{
    return guarded([&] {
        if(!p || !target || n < 0 || (n > 0 && (!ic || !T || !output)))
            throw std::invalid_argument("integrateOrbitsTargetMany: invalid arguments");
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(p->pot->device));
        const size_t m = static_cast<size_t>(n) * target->numValues;
        DevBuf<double> dic(6 * n), dT(n), dout(6 * n);
        DevBuf<float> dres(m);
        DevBuf<long> dsteps(n);
        DevBuf<int> dstat(n);
        AGB_CUDA(cudaMemcpy(dic.ptr, ic, 6 * n * sizeof(double), cudaMemcpyHostToDevice));
        AGB_CUDA(cudaMemcpy(dT.ptr, T, n * sizeof(double), cudaMemcpyHostToDevice));
        if(agama_integrateOrbitsTargetManyDevice(p, n, dic.ptr, dT.ptr, Omega, accuracy, maxNumSteps, target,
                dres.ptr, dout.ptr, dsteps.ptr, dstat.ptr, nullptr) != 0)
            throw std::runtime_error(lastError());
        AGB_CUDA(cudaMemcpy(output, dres.ptr, m * sizeof(float), cudaMemcpyDeviceToHost));
        if(finalState) AGB_CUDA(cudaMemcpy(finalState, dout.ptr, 6 * n * sizeof(double), cudaMemcpyDeviceToHost));
        if(numSteps) AGB_CUDA(cudaMemcpy(numSteps, dsteps.ptr, n * sizeof(long), cudaMemcpyDeviceToHost));
        if(status) AGB_CUDA(cudaMemcpy(status, dstat.ptr, n * sizeof(int), cudaMemcpyDeviceToHost));
    });
}

// ---- orbit batches captured once in a CUDA graph and replayed

struct agama_OrbitGraph {
    int device = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    DevBuf<unsigned long long> queue;
    OrbitShape shape;
    ~agama_OrbitGraph() {
        if(exec) cudaGraphExecDestroy(exec);
        if(graph) cudaGraphDestroy(graph);
    }
};

extern "C" agama_OrbitGraph* agama_orbitGraphCreate(const agama_Potential* p, long n, const double* ic,
    const double* T, double Omega, double accuracy, long maxNumSteps, double* finalState, long* numSteps,
    long* numRejected, int* status)
{
    CurrentDeviceGuard keep;
    try {
        if(!p || n <= 0 || !ic || !T || !finalState) throw std::invalid_argument("orbitGraphCreate: invalid arguments");
        AGB_CUDA(cudaSetDevice(p->pot->device));
        const OrbitParams P = makeOrbitParams(Omega, accuracy, maxNumSteps);
        agama_OrbitGraph* g = new agama_OrbitGraph;
        try {
            g->device = p->pot->device;
            g->queue.alloc(1);
            cudaStream_t s;
            AGB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
            // the launch shape is settled (autotuner trial) before the capture begins
            g->shape = orbitShapeFor(p->pot->view, P, n, ic, T, s);
            AGB_CUDA(cudaStreamSynchronize(s));
            AGB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            launchOrbits(p->pot->view, P, n, ic, T, finalState, numSteps, numRejected, status, g->queue.ptr, s,
                g->shape);
            AGB_CUDA(cudaStreamEndCapture(s, &g->graph));
            AGB_CUDA(cudaGraphInstantiate(&g->exec, g->graph, 0));
            AGB_CUDA(cudaStreamDestroy(s));
        } catch(...) {
            delete g;
            throw;
        }
        return g;
    } catch(std::exception& e) {
        setError(e.what());
        return nullptr;
    }
}

extern "C" int agama_orbitGraphLaunch(agama_OrbitGraph* g, void* stream)
{
    return guarded([&] {
        if(!g) throw std::invalid_argument("orbitGraphLaunch: null graph");
        AGB_CUDA(cudaSetDevice(g->device));
        AGB_CUDA(cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream)));
    });
}

extern "C" int agama_orbitGraphLanes(const agama_OrbitGraph* g) { return g ? g->shape.lanes : 0; }
extern "C" int agama_orbitGraphBlockSize(const agama_OrbitGraph* g) { return g ? g->shape.block : 0; }

extern "C" void agama_orbitGraphDelete(agama_OrbitGraph* g) { delete g; }

extern "C" int agama_integrateOrbitsMany(const agama_Potential* p, long n, const double* ic,
    const double* T, double Omega, double accuracy, long maxNumSteps, double* finalState,
    long* numSteps, int* status)
{
    return guarded([&] {
        if(!p || n < 0 || (n > 0 && (!ic || !T || !finalState)))
            throw std::invalid_argument("integrateOrbitsMany: invalid arguments");
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(p->pot->device));
        const OrbitParams P = makeOrbitParams(Omega, accuracy, maxNumSteps);
        DevBuf<double> dic(6 * n), dT(n), dout(6 * n);
        DevBuf<long> dsteps(n);
        DevBuf<int> dstat(n);
        DevBuf<unsigned long long> q(1);
        AGB_CUDA(cudaMemcpy(dic.ptr, ic, 6 * n * sizeof(double), cudaMemcpyHostToDevice));
        AGB_CUDA(cudaMemcpy(dT.ptr, T, n * sizeof(double), cudaMemcpyHostToDevice));
        launchOrbits(p->pot->view, P, n, dic.ptr, dT.ptr, dout.ptr, dsteps.ptr, nullptr, dstat.ptr, q.ptr, 0);
        AGB_CUDA(cudaMemcpy(finalState, dout.ptr, 6 * n * sizeof(double), cudaMemcpyDeviceToHost));
        if(numSteps) AGB_CUDA(cudaMemcpy(numSteps, dsteps.ptr, n * sizeof(long), cudaMemcpyDeviceToHost));
        if(status) AGB_CUDA(cudaMemcpy(status, dstat.ptr, n * sizeof(int), cudaMemcpyDeviceToHost));
    });
}

extern "C" int agama_integrateOrbitsManyDeviceNoAlloc(const agama_Potential* p, long n, const double* ic,
    const double* T, double Omega, double accuracy, long maxNumSteps, double* finalState,
    long* numSteps, long* numRejected, int* status, int queueSlot, void* stream)
{
    // no cudaMalloc / cudaFree / allocating library call on this path: the work-queue counter is
    // a slot of the library's static device array (launchOrbitsNoAlloc, orbit.cu)
    return guarded([&] {
        if(!p || n < 0 || (n > 0 && (!ic || !T || !finalState)))
            throw std::invalid_argument("integrateOrbitsManyDeviceNoAlloc: invalid arguments");
        if(queueSlot < 0 || queueSlot >= noallocQueueSlots())
            throw std::invalid_argument("integrateOrbitsManyDeviceNoAlloc: queueSlot " + std::to_string(queueSlot) +
                " out of range 0.." + std::to_string(noallocQueueSlots() - 1));
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(p->pot->device));
        const OrbitParams P = makeOrbitParams(Omega, accuracy, maxNumSteps);
        launchOrbitsNoAlloc(p->pot->view, P, n, ic, T, finalState, numSteps, numRejected, status, queueSlot,
            static_cast<cudaStream_t>(stream));
    });
}

// ------------------------------------------------------------------------------------------
// actions (Staeckel fudge)

struct agama_ActionFinder { DeviceActionFinder* af; };

namespace {
void requireAxisymmetric(const agama_Potential* p) {
    if(!p) throw std::invalid_argument("null potential");
    if(!p->pot->axisymmetric)
        throw std::invalid_argument("Fudge approximation only works for axisymmetric potentials");
}
std::vector<double> vec(const double* p, long n) { return p ? std::vector<double>(p, p + n) : std::vector<double>(); }
}  // namespace

extern "C" agama_ActionFinder* agama_createActionFinderFromTables(const agama_Potential* p,
    int nE, const double* gridE, int nL, const double* gridL, const double* delta,
    int nLofE, const double* LofE, int nRofL, const double* RofL, int nPhiofR, const double* PhiofR,
    const double* scalars)
{
    CurrentDeviceGuard keep;
    try {
        requireAxisymmetric(p);
        if(nE < 2 || nL < 2 || !gridE || !gridL || !delta || nLofE < 2 || !LofE || nRofL < 2 || !RofL ||
            nPhiofR < 2 || !PhiofR || !scalars)
            throw std::invalid_argument("createActionFinderFromTables: invalid arguments");
        AGB_CUDA(cudaSetDevice(p->pot->device));
        FinderTablesHost T;
        T.nE = nE; T.nL = nL;
        T.gridE = vec(gridE, nE); T.gridL = vec(gridL, nL); T.delta = vec(delta, static_cast<long>(nE) * nL);
        T.lofe = vec(LofE, 4L * nLofE); T.rofl = vec(RofL, 4L * nRofL); T.phiofr = vec(PhiofR, 4L * nPhiofR);
        T.invPhi0 = scalars[0]; T.interpInvPhi0 = scalars[1]; T.slopeOut = scalars[2];
        T.coefOut = scalars[3]; T.massOut = scalars[4];
        return new agama_ActionFinder{ createDeviceActionFinder(p->pot, T) };
    } catch(std::exception& e) {
        setError(e.what());
        return nullptr;
    }
}

extern "C" agama_ActionFinder* agama_createActionFinder(const agama_Potential* p)
{
    CurrentDeviceGuard keep;
    try {
        requireAxisymmetric(p);
        AGB_CUDA(cudaSetDevice(p->pot->device));
        return new agama_ActionFinder{ createDeviceActionFinder(p->pot, buildFinderTables(*p->pot)) };
    } catch(std::exception& e) {
        setError(e.what());
        return nullptr;
    }
}

extern "C" int agama_getActionFinderTableSizes(const agama_ActionFinder* a, int* nE, int* nL, int* nLofE,
    int* nRofL, int* nPhiofR)
{
    return guarded([&] {
        if(!a) throw std::invalid_argument("null action finder");
        const FinderTablesHost& T = a->af->host;
        if(nE) *nE = T.nE;
        if(nL) *nL = T.nL;
        if(nLofE) *nLofE = static_cast<int>(T.lofe.size() / 4);
        if(nRofL) *nRofL = static_cast<int>(T.rofl.size() / 4);
        if(nPhiofR) *nPhiofR = static_cast<int>(T.phiofr.size() / 4);
    });
}

extern "C" int agama_getActionFinderTables(const agama_ActionFinder* a, double* gridE, double* gridL,
    double* delta, double* LofE, double* RofL, double* PhiofR, double* scalars)
{
    return guarded([&] {
        if(!a) throw std::invalid_argument("null action finder");
        const FinderTablesHost& T = a->af->host;
        auto put = [](const std::vector<double>& v, double* out) { if(out) std::copy(v.begin(), v.end(), out); };
        put(T.gridE, gridE); put(T.gridL, gridL); put(T.delta, delta);
        put(T.lofe, LofE); put(T.rofl, RofL); put(T.phiofr, PhiofR);
        if(scalars) {
            scalars[0] = T.invPhi0; scalars[1] = T.interpInvPhi0; scalars[2] = T.slopeOut;
            scalars[3] = T.coefOut; scalars[4] = T.massOut;
        }
    });
}

extern "C" void agama_deleteActionFinder(agama_ActionFinder* a)
{
    if(!a) return;
    delete a->af;
    delete a;
}

namespace {
/// the bracket predictor of a finder when it is switched on, and its search counters (null when no
/// predictor was ever trained)
const BracketPlan* planOf(const DeviceActionFinder& F, BracketPlan& tmp)
{
    if(!F.bracketStats.ptr) return nullptr;     // no predictor trained: plain searches, no counters
    tmp.net = F.useBrackets ? F.brackets : nullptr;
    for(int k = 0; k < 3; k++) tmp.widths[k] = F.bracketWidths[k];
    tmp.stats = F.countBrackets ? F.bracketStats.ptr : nullptr;
    if(!tmp.net && !tmp.stats) return nullptr;  // plain searches without counters
    return &tmp;
}
}  // namespace

extern "C" int agama_evalActionsAnglesFrequenciesManyDevice(const agama_ActionFinder* a, long n,
    const double* posvel, double* act, double* ang, double* freq, void* stream)
{
    return guarded([&] {
        if(!a || n < 0 || (n > 0 && (!posvel || !(act || ang || freq))))
            throw std::invalid_argument("evalActionsAnglesFrequenciesManyDevice: invalid arguments");
        AGB_CUDA(cudaSetDevice(a->af->pot->device));
        BracketPlan plan;
        launchActionsFinder(a->af->pot->view, a->af->view, n, posvel, act, ang, freq, nullptr, nullptr,
            static_cast<cudaStream_t>(stream), planOf(*a->af, plan));
    });
}

extern "C" int agama_evalActionsAnglesFrequenciesMany(const agama_ActionFinder* a, long n,
    const double* posvel, double* act, double* ang, double* freq)
{
    return guarded([&] {
        if(!a || n < 0 || (n > 0 && (!posvel || !(act || ang || freq))))
            throw std::invalid_argument("evalActionsAnglesFrequenciesMany: invalid arguments");
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(a->af->pot->device));
        const DeviceActionFinder& F = *a->af;
        runChunked(n, { { posvel, 6 * sizeof(double) } },
            { { act, 3 * sizeof(double) }, { ang, 3 * sizeof(double) }, { freq, 3 * sizeof(double) } },
            [&](long, long count, void* const* in, void* const* out, cudaStream_t s) {
                BracketPlan plan;
                launchActionsFinder(F.pot->view, F.view, count, static_cast<const double*>(in[0]),
                    static_cast<double*>(out[0]), static_cast<double*>(out[1]), static_cast<double*>(out[2]),
                    nullptr, nullptr, s, planOf(F, plan));
            });
    });
}

extern "C" int agama_evalActionsManyDevice(const agama_ActionFinder* a, long n, const double* posvel,
    double* act, double* fdOut, void* stream)
{
    return guarded([&] {
        if(!a || n < 0 || (n > 0 && (!posvel || !act))) throw std::invalid_argument("evalActionsManyDevice: invalid arguments");
        AGB_CUDA(cudaSetDevice(a->af->pot->device));
        BracketPlan plan;
        launchActionsFinder(a->af->pot->view, a->af->view, n, posvel, act, nullptr, nullptr, fdOut, nullptr,
            static_cast<cudaStream_t>(stream), planOf(*a->af, plan));
    });
}

extern "C" int agama_evalActionsMany(const agama_ActionFinder* a, long n, const double* posvel,
    double* act, double* fdOut)
{
    return guarded([&] {
        if(!a || n < 0 || (n > 0 && (!posvel || !act))) throw std::invalid_argument("evalActionsMany: invalid arguments");
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(a->af->pot->device));
        const DeviceActionFinder& F = *a->af;
        runChunked(n, { { posvel, 6 * sizeof(double) } }, { { act, 3 * sizeof(double) }, { fdOut, sizeof(double) } },
            [&](long, long count, void* const* in, void* const* out, cudaStream_t s) {
                BracketPlan plan;
                launchActionsFinder(F.pot->view, F.view, count, static_cast<const double*>(in[0]),
                    static_cast<double*>(out[0]), nullptr, nullptr, static_cast<double*>(out[1]), nullptr, s,
                    planOf(F, plan));
            });
    });
}

extern "C" int agama_evalActionsAnglesFrequenciesStandaloneManyDevice(const agama_Potential* p, long n,
    const double* posvel, const double* fd, double fd0, double* act, double* ang, double* freq, void* stream)
{
    return guarded([&] {
        requireAxisymmetric(p);
        if(n < 0 || (n > 0 && (!posvel || !(act || ang || freq))))
            throw std::invalid_argument("evalActionsAnglesFrequenciesStandaloneManyDevice: invalid arguments");
        AGB_CUDA(cudaSetDevice(p->pot->device));
        launchActionsFixedDelta(p->pot->view, n, posvel, fd, fd0, act, ang, freq, nullptr,
            static_cast<cudaStream_t>(stream));
    });
}

extern "C" int agama_evalActionsAnglesFrequenciesStandaloneMany(const agama_Potential* p, long n,
    const double* posvel, const double* fd, double fd0, double* act, double* ang, double* freq)
{
    return guarded([&] {
        requireAxisymmetric(p);
        if(n < 0 || (n > 0 && (!posvel || !(act || ang || freq))))
            throw std::invalid_argument("evalActionsAnglesFrequenciesStandaloneMany: invalid arguments");
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(p->pot->device));
        const MultipoleView& M = p->pot->view;
        runChunked(n, { { posvel, 6 * sizeof(double) }, { fd, sizeof(double) } },
            { { act, 3 * sizeof(double) }, { ang, 3 * sizeof(double) }, { freq, 3 * sizeof(double) } },
            [&](long, long count, void* const* in, void* const* out, cudaStream_t s) {
                launchActionsFixedDelta(M, count, static_cast<const double*>(in[0]), static_cast<const double*>(in[1]),
                    fd0, static_cast<double*>(out[0]), static_cast<double*>(out[1]), static_cast<double*>(out[2]),
                    nullptr, s);
            });
    });
}

extern "C" int agama_evalActionsStandaloneManyDevice(const agama_Potential* p, long n, const double* posvel,
    const double* fd, double fd0, double* act, int* rootIters, void* stream)
{
    return guarded([&] {
        requireAxisymmetric(p);
        if(n < 0 || (n > 0 && (!posvel || !act))) throw std::invalid_argument("evalActionsStandaloneManyDevice: invalid arguments");
        AGB_CUDA(cudaSetDevice(p->pot->device));
        launchActionsFixedDelta(p->pot->view, n, posvel, fd, fd0, act, nullptr, nullptr, rootIters,
            static_cast<cudaStream_t>(stream));
    });
}

extern "C" int agama_evalActionsStandaloneMany(const agama_Potential* p, long n, const double* posvel,
    const double* fd, double fd0, double* act)
{
    return guarded([&] {
        requireAxisymmetric(p);
        if(n < 0 || (n > 0 && (!posvel || !act))) throw std::invalid_argument("evalActionsStandaloneMany: invalid arguments");
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(p->pot->device));
        const MultipoleView& M = p->pot->view;
        runChunked(n, { { posvel, 6 * sizeof(double) }, { fd, sizeof(double) } }, { { act, 3 * sizeof(double) } },
            [&](long, long count, void* const* in, void* const* out, cudaStream_t s) {
                launchActionsFixedDelta(M, count, static_cast<const double*>(in[0]), static_cast<const double*>(in[1]),
                    fd0, static_cast<double*>(out[0]), nullptr, nullptr, nullptr, s);
            });
    });
}

namespace {
/// the single-point outputs of the reference's C interface: NaN everywhere when the call failed
void storeSinglePoint(int rc, const double* act, const double* ang, const double* freq,
    double actions[3], double angles[3], double frequencies[3])
{
    for(int k = 0; k < 3; k++) {
        if(actions) actions[k] = rc == 0 ? act[k] : NAN;
        if(angles) angles[k] = rc == 0 ? ang[k] : NAN;
        if(frequencies) frequencies[k] = rc == 0 ? freq[k] : NAN;
    }
}
}  // namespace

extern "C" void agama_evalActionsAnglesFrequencies(const agama_ActionFinder* a, const double posvel[6],
    double actions[3], double angles[3], double frequencies[3])
{
    double act[3], ang[3], freq[3];
    const int rc = agama_evalActionsAnglesFrequenciesMany(a, 1, posvel, act, angles ? ang : nullptr,
        frequencies ? freq : nullptr);
    storeSinglePoint(rc, act, ang, freq, actions, angles, frequencies);
}

extern "C" void agama_evalActionsAnglesFrequenciesStandalone(const agama_Potential* p, double fd,
    const double posvel[6], double actions[3], double angles[3], double frequencies[3])
{
    double act[3], ang[3], freq[3];
    const int rc = agama_evalActionsAnglesFrequenciesStandaloneMany(p, 1, posvel, nullptr, fd, act,
        angles ? ang : nullptr, frequencies ? freq : nullptr);
    storeSinglePoint(rc, act, ang, freq, actions, angles, frequencies);
}

extern "C" int agama_gemmBf16Device(int M, int N, int K, const void* A, const void* B, float* C, int ldc,
    int accumulate, void* stream)
{
    return guarded([&] {
        if(M < 0 || N < 0 || K < 0 || (M > 0 && N > 0 && K > 0 && (!A || !B || !C)))
            throw std::invalid_argument("gemmBf16Device: invalid arguments");
        requireDevice();
        // a workspace for the split-K form of outputs with few tiles (released in stream order)
        const size_t wsFloats = static_cast<size_t>(16) * M * N;
        const bool few = M > 0 && N > 0 && (M / 128) * (N / 128) <= 32;
        Scratch ws(few ? wsFloats * sizeof(float) : 256, static_cast<cudaStream_t>(stream));
        launchGemmBf16(M, N, K, A, B, C, ldc, accumulate != 0, static_cast<cudaStream_t>(stream),
            few ? static_cast<float*>(ws.ptr) : nullptr, few ? wsFloats : 0);
    });
}

// ------------------------------------------------------------------------------------------
// the bracket predictor of an action finder

extern "C" int agama_actionFinderBracketSamples(const agama_ActionFinder* a, long n, const double* posvel,
    float* features, float* target, float* mask)
{
    return guarded([&] {
        if(!a || n <= 0 || !posvel || !features || !target || !mask)
            throw std::invalid_argument("actionFinderBracketSamples: invalid arguments");
        AGB_CUDA(cudaSetDevice(a->af->pot->device));
        DevBuf<double> dpv(6 * n);
        DevBuf<float> f(6 * n), t(3 * n), m(3 * n);
        AGB_CUDA(cudaMemcpy(dpv.ptr, posvel, sizeof(double) * 6 * n, cudaMemcpyHostToDevice));
        launchBracketSamples(a->af->pot->view, a->af->view, n, dpv.ptr, BracketSamples{ f.ptr, t.ptr, m.ptr }, 0);
        AGB_CUDA(cudaMemcpy(features, f.ptr, sizeof(float) * 6 * n, cudaMemcpyDeviceToHost));
        AGB_CUDA(cudaMemcpy(target, t.ptr, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost));
        AGB_CUDA(cudaMemcpy(mask, m.ptr, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost));
    });
}

extern "C" int agama_actionFinderTrainBrackets(agama_ActionFinder* a, long n, const double* posvel, int epochs,
    int batch, float lr, unsigned long long seed, float* lossHistory, float* widths)
{
    return guarded([&] {
        if(!a || n < 1024 || !posvel || epochs < 1) throw std::invalid_argument("actionFinderTrainBrackets: invalid arguments");
        DeviceActionFinder& F = *a->af;
        AGB_CUDA(cudaSetDevice(F.pot->device));
        // inputs and targets of every sample from the plain root searches
        DevBuf<double> dpv(6 * n);
        DevBuf<float> f(6 * n), t(3 * n), m(3 * n);
        AGB_CUDA(cudaMemcpy(dpv.ptr, posvel, sizeof(double) * 6 * n, cudaMemcpyHostToDevice));
        launchBracketSamples(F.pot->view, F.view, n, dpv.ptr, BracketSamples{ f.ptr, t.ptr, m.ptr }, 0);
        AGB_CUDA(cudaDeviceSynchronize());
        // train on the first 90 %, size the brackets on the held-out 10 %
        const long nVal = std::max(128L, n / 10), nTrain = n - nVal;
        Mlp* net = new Mlp(seed);
        try {
            const std::vector<float> hist = net->train(nTrain, f.ptr, t.ptr, m.ptr, epochs, batch, lr, seed + 1, 0);
            if(lossHistory) for(size_t k = 0; k < hist.size(); k++) lossHistory[k] = hist[k];
            DevBuf<float> y(3 * nVal);
            net->predict(nVal, f.ptr + 6 * nTrain, y.ptr, 0);
            AGB_CUDA(cudaDeviceSynchronize());
            net->checkError();
            std::vector<float> hy(3 * nVal), ht(3 * nVal), hm(3 * nVal);
            AGB_CUDA(cudaMemcpy(hy.data(), y.ptr, sizeof(float) * 3 * nVal, cudaMemcpyDeviceToHost));
            AGB_CUDA(cudaMemcpy(ht.data(), t.ptr + 3 * nTrain, sizeof(float) * 3 * nVal, cudaMemcpyDeviceToHost));
            AGB_CUDA(cudaMemcpy(hm.data(), m.ptr + 3 * nTrain, sizeof(float) * 3 * nVal, cudaMemcpyDeviceToHost));
            float w[3];
            for(int k = 0; k < 3; k++) {
                // half-width: twice the 95th percentile of the held-out error (at least 1e-4): the
                // few percent of searches that miss fall back to the plain bracket
                std::vector<float> e;
                for(long i = 0; i < nVal; i++)
                    if(hm[3 * i + k] > 0 && std::isfinite(hy[3 * i + k])) e.push_back(std::fabs(hy[3 * i + k] - ht[3 * i + k]));
                float q = 1;
                if(!e.empty()) {
                    const size_t at = std::min(e.size() - 1, static_cast<size_t>(0.95 * e.size()));
                    std::nth_element(e.begin(), e.begin() + at, e.end());
                    q = e[at];
                }
                w[k] = std::max(2 * q, 1e-4f);
            }
            delete F.brackets;
            F.brackets = net;
            for(int k = 0; k < 3; k++) F.bracketWidths[k] = w[k];
            if(widths) for(int k = 0; k < 3; k++) widths[k] = w[k];
            F.useBrackets = true;
            if(!F.bracketStats.ptr) F.bracketStats.alloc(4);
            AGB_CUDA(cudaMemset(F.bracketStats.ptr, 0, 4 * sizeof(unsigned long long)));
        } catch(...) {
            delete net;
            throw;
        }
    });
}

extern "C" int agama_actionFinderPredictBrackets(const agama_ActionFinder* a, long n, const float* features,
    float* prediction)
{
    return guarded([&] {
        if(!a || n < 0 || (n > 0 && (!features || !prediction)))
            throw std::invalid_argument("actionFinderPredictBrackets: invalid arguments");
        if(!a->af->brackets) throw std::invalid_argument("actionFinderPredictBrackets: no bracket predictor trained");
        if(n == 0) return;
        AGB_CUDA(cudaSetDevice(a->af->pot->device));
        DevBuf<float> f(6 * n), y(3 * n);
        AGB_CUDA(cudaMemcpy(f.ptr, features, sizeof(float) * 6 * n, cudaMemcpyHostToDevice));
        a->af->brackets->predict(n, f.ptr, y.ptr, 0);
        AGB_CUDA(cudaMemcpy(prediction, y.ptr, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost));
        a->af->brackets->checkError();
    });
}

extern "C" int agama_actionFinderUseBrackets(agama_ActionFinder* a, int on)
{
    return guarded([&] {
        if(!a) throw std::invalid_argument("actionFinderUseBrackets: null finder");
        if(on && !a->af->brackets) throw std::invalid_argument("actionFinderUseBrackets: no bracket predictor trained");
        a->af->useBrackets = on != 0;
    });
}

extern "C" int agama_actionFinderCountBrackets(agama_ActionFinder* a, int on)
{
    return guarded([&] {
        if(!a) throw std::invalid_argument("actionFinderCountBrackets: null finder");
        a->af->countBrackets = on != 0;
    });
}

extern "C" int agama_actionFinderBracketStats(agama_ActionFinder* a, long long* stats, int reset)
{
    return guarded([&] {
        if(!a || !stats) throw std::invalid_argument("actionFinderBracketStats: invalid arguments");
        DeviceActionFinder& F = *a->af;
        unsigned long long h[4] = { 0, 0, 0, 0 };
        if(F.bracketStats.ptr) {
            AGB_CUDA(cudaSetDevice(F.pot->device));
            AGB_CUDA(cudaDeviceSynchronize());
            AGB_CUDA(cudaMemcpy(h, F.bracketStats.ptr, sizeof(h), cudaMemcpyDeviceToHost));
            if(reset) AGB_CUDA(cudaMemset(F.bracketStats.ptr, 0, sizeof(h)));
        }
        for(int k = 0; k < 4; k++) stats[k] = static_cast<long long>(h[k]);
    });
}

// ------------------------------------------------------------------------------------------
// the bracket-predictor network

struct agama_Mlp { Mlp* net; };

extern "C" agama_Mlp* agama_mlpCreate(unsigned long long seed)
{
    try {
        requireDevice();
        return new agama_Mlp{ new Mlp(seed) };
    } catch(std::exception& e) {
        setError(e.what());
        return nullptr;
    }
}

extern "C" void agama_mlpDelete(agama_Mlp* m)
{
    if(!m) return;
    delete m->net;
    delete m;
}

extern "C" int agama_mlpNumParams() { return MLP_NUM_PARAMS; }

extern "C" int agama_mlpGetParams(const agama_Mlp* m, float* params, float* scaling)
{
    return guarded([&] {
        if(!m) throw std::invalid_argument("mlpGetParams: null network");
        AGB_CUDA(cudaSetDevice(m->net->device));
        if(params) AGB_CUDA(cudaMemcpy(params, m->net->params.ptr, sizeof(float) * MLP_NUM_PARAMS, cudaMemcpyDeviceToHost));
        if(scaling) AGB_CUDA(cudaMemcpy(scaling, m->net->scaling.ptr, sizeof(float) * 18, cudaMemcpyDeviceToHost));
    });
}

extern "C" int agama_mlpSetParams(agama_Mlp* m, const float* params, const float* scaling)
{
    return guarded([&] {
        if(!m) throw std::invalid_argument("mlpSetParams: null network");
        AGB_CUDA(cudaSetDevice(m->net->device));
        if(params) AGB_CUDA(cudaMemcpy(m->net->params.ptr, params, sizeof(float) * MLP_NUM_PARAMS, cudaMemcpyHostToDevice));
        if(scaling) AGB_CUDA(cudaMemcpy(m->net->scaling.ptr, scaling, sizeof(float) * 18, cudaMemcpyHostToDevice));
        m->net->refreshWeights(0);
        AGB_CUDA(cudaDeviceSynchronize());
    });
}

extern "C" int agama_mlpLossGrad(agama_Mlp* m, int batch, const float* x, const float* t, const float* mask,
    float* grad, float* loss)
{
    return guarded([&] {
        if(!m || !x || !t || !mask || !grad) throw std::invalid_argument("mlpLossGrad: invalid arguments");
        AGB_CUDA(cudaSetDevice(m->net->device));
        DevBuf<float> g(MLP_NUM_PARAMS);
        const float l = m->net->lossGradDevice(batch, x, t, mask, g.ptr, 0);
        AGB_CUDA(cudaMemcpy(grad, g.ptr, sizeof(float) * MLP_NUM_PARAMS, cudaMemcpyDeviceToHost));
        if(loss) *loss = l;
    });
}

extern "C" int agama_mlpTrain(agama_Mlp* m, long n, const float* x, const float* t, const float* mask, int epochs,
    int batch, float lr, unsigned long long seed, float* lossHistory)
{
    return guarded([&] {
        if(!m || n <= 0 || !x || !t || !mask || epochs < 0) throw std::invalid_argument("mlpTrain: invalid arguments");
        AGB_CUDA(cudaSetDevice(m->net->device));
        const std::vector<float> h = m->net->train(n, x, t, mask, epochs, batch, lr, seed, 0);
        if(lossHistory) for(size_t k = 0; k < h.size(); k++) lossHistory[k] = h[k];
    });
}

extern "C" int agama_mlpPredictDevice(const agama_Mlp* m, long n, const float* x, float* y, void* stream)
{
    return guarded([&] {
        if(!m || n < 0 || (n > 0 && (!x || !y))) throw std::invalid_argument("mlpPredictDevice: invalid arguments");
        AGB_CUDA(cudaSetDevice(m->net->device));
        m->net->predict(n, x, y, static_cast<cudaStream_t>(stream));
    });
}

extern "C" int agama_mlpCheck(const agama_Mlp* m)
{
    return guarded([&] {
        if(!m) throw std::invalid_argument("mlpCheck: null network");
        AGB_CUDA(cudaSetDevice(m->net->device));
        AGB_CUDA(cudaDeviceSynchronize());
        m->net->checkError();
    });
}

// ------------------------------------------------------------------------------------------
// device FP64 throughput probe (the roofline denominator for the FP64-bound kernels)

namespace {
__global__ void fp64FmaProbe(double* out, int iters)
{
    // 8 independent FMA chains per thread keep the FP64 pipe busy
    double a[8];
    const double b = 1.0000001, c = 1e-9;
    for(int k = 0; k < 8; k++) a[k] = threadIdx.x * 1e-7 + k;
    for(int i = 0; i < iters; i++)
#pragma unroll
        for(int k = 0; k < 8; k++) a[k] = fma(a[k], b, c);
    double s = 0;
    for(int k = 0; k < 8; k++) s += a[k];
    if(s == 12345.678) out[0] = s;   // keeps the chains live
}
}  // namespace

extern "C" int agama_actionPhaseTiming(int on, double* ms, long* passes)
{
    return guarded([&] { setActionPhaseTiming(on != 0, ms, passes); });
}

extern "C" int agama_measureFP64Throughput(double* tflops)
{
    return guarded([&] {
        requireDevice();
        int dev, sms;
        AGB_CUDA(cudaGetDevice(&dev));
        AGB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        DevBuf<double> out(1);
        const int block = 256, grid = sms * 8, iters = 4096;
        cudaEvent_t e0, e1;
        AGB_CUDA(cudaEventCreate(&e0));
        AGB_CUDA(cudaEventCreate(&e1));
        fp64FmaProbe<<<grid, block>>>(out.ptr, iters);   // warm-up
        float best = 1e30f;
        for(int rep = 0; rep < 5; rep++) {
            AGB_CUDA(cudaEventRecord(e0));
            fp64FmaProbe<<<grid, block>>>(out.ptr, iters);
            AGB_CUDA(cudaEventRecord(e1));
            AGB_CUDA(cudaEventSynchronize(e1));
            float ms;
            AGB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            best = std::min(best, ms);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *tflops = 2.0 * 8 * iters * static_cast<double>(grid) * block / (best * 1e-3) / 1e12;
    });
}
