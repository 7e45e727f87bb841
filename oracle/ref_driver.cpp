// Flat C API over the reference Agama library, compiled from the reference sources into
// oracle/_ref/libagama_ref.so.  TEST INFRASTRUCTURE ONLY: used by tests/, by the fixture
// generator and by the CPU reference arm of bench.py -- never by the engine itself.
//
// Each loop mirrors the way the reference's own Python binding drives the library:
//   potential / force : OpenMP dynamic chunks of 1024 points  (interface_python.cpp:1405-1485)
//   orbits            : OpenMP schedule(dynamic,1) over orbits (interface_python.cpp:8101)
//   actions           : OpenMP dynamic chunks of 64 points     (interface_python.cpp:3791-3822)
// and calls the same library entry points:
//   BasePotential::eval(PosCar)                 potential_base.h:153-156
//   orbit::OrbitIntegrator<Car>::init/run       orbit.cpp:52-117
//   actions::ActionFinderAxisymFudge::eval      actions_staeckel.cpp:954-979
//   actions::evalAxisymFudge (fixed Delta)      actions_staeckel.cpp:683-693
// The table-export functions read private members of the action finder so that the exact
// focal-distance table and L_circ(E) spline used by the reference can be handed to tests.
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include <algorithm>
#include <omp.h>
// expose the private interpolation tables of the action finder (test code only)
#define private public
#define protected public
#include "actions_staeckel.h"
#include "potential_utils.h"
#include "math_spline.h"
#include "math_core.h"
#include "math_sphharm.h"
#undef private
#undef protected
#include "potential_factory.h"
#include "potential_composite.h"
#include "potential_multipole.h"
#include "potential_base.h"
#include "orbit.h"
#include "coord.h"
#include "utils.h"

namespace {

std::string g_error;

void setThreads(int nthreads) { if(nthreads > 0) omp_set_num_threads(nthreads); }

/// forwarding potential that counts evaluations (pattern of SPotential in the reference's
/// tests/test_potential_expansions.cpp:289-302)
class CountingPotential: public potential::BasePotential {
public:
    potential::PtrPotential pot;
    mutable std::atomic<long long> count;
    explicit CountingPotential(const potential::PtrPotential& p) : pot(p), count(0) {}
    virtual coord::SymmetryType symmetry() const { return pot->symmetry(); }
    virtual std::string name() const { return pot->name(); }
protected:
    virtual void evalCar(const coord::PosCar &pos, double* p, coord::GradCar* g, coord::HessCar* h, double t) const
    { ++count; pot->eval(pos, p, g, h, t); }
    virtual void evalCyl(const coord::PosCyl &pos, double* p, coord::GradCyl* g, coord::HessCyl* h, double t) const
    { ++count; pot->eval(pos, p, g, h, t); }
    virtual void evalSph(const coord::PosSph &pos, double* p, coord::GradSph* g, coord::HessSph* h, double t) const
    { ++count; pot->eval(pos, p, g, h, t); }
    virtual double densityCar(const coord::PosCar &pos, double t) const { return pot->density(pos, t); }
    virtual double densityCyl(const coord::PosCyl &pos, double t) const { return pot->density(pos, t); }
    virtual double densitySph(const coord::PosSph &pos, double t) const { return pot->density(pos, t); }
};

struct PotHandle { potential::PtrPotential pot; };
struct AfHandle  { std::shared_ptr<CountingPotential> cnt; std::shared_ptr<actions::ActionFinderAxisymFudge> af; };

/// runtime function counting accepted DOP853 steps
class StepCounter: public orbit::BaseRuntimeFnc {
public:
    long* counter;
    StepCounter(orbit::BaseOrbitIntegrator& o, long* c) : orbit::BaseRuntimeFnc(o), counter(c) {}
    virtual bool processTimestep(double, double) { ++*counter; return true; }
};

}  // namespace

extern "C" {

const char* ref_error() { return g_error.c_str(); }

/// load a potential from an INI file (e.g. a Multipole coefficient file written by writePotential)
void* ref_load_potential(const char* iniFile) {
    try {
        PotHandle* h = new PotHandle;
        h->pot = potential::readPotential(iniFile);
        return h;
    } catch(std::exception& e) { g_error = e.what(); return NULL; }
}

/// create a potential from key=value parameters (as agama_createPotential does)
void* ref_create_potential(const char* params) {
    try {
        PotHandle* h = new PotHandle;
        h->pot = potential::createPotential(utils::KeyValueMap(std::string(params)));
        return h;
    } catch(std::exception& e) { g_error = e.what(); return NULL; }
}

int ref_write_potential(void* pot, const char* file) {
    try { return potential::writePotential(file, *static_cast<PotHandle*>(pot)->pot) ? 0 : -1; }
    catch(std::exception& e) { g_error = e.what(); return -1; }
}

void ref_free_potential(void* pot) { delete static_cast<PotHandle*>(pot); }

/// potential, gradient (dPhi/dx) and optional Hessian (xx,yy,zz,xy,yz,zx) at n Cartesian points
int ref_eval_many(void* handle, long n, const double* pos, double* phi, double* grad, double* hess, int nthreads) {
    const potential::BasePotential& pot = *static_cast<PotHandle*>(handle)->pot;
    setThreads(nthreads);
    std::string err;
#pragma omp parallel for schedule(dynamic, 1024)
    for(long i = 0; i < n; i++) {
        try {
            double p; coord::GradCar g; coord::HessCar h;
            pot.eval(coord::PosCar(pos[3*i], pos[3*i+1], pos[3*i+2]), &p, grad ? &g : NULL, hess ? &h : NULL);
            if(phi) phi[i] = p;
            if(grad) { grad[3*i] = g.dx; grad[3*i+1] = g.dy; grad[3*i+2] = g.dz; }
            if(hess) { hess[6*i] = h.dx2; hess[6*i+1] = h.dy2; hess[6*i+2] = h.dz2;
                       hess[6*i+3] = h.dxdy; hess[6*i+4] = h.dydz; hess[6*i+5] = h.dxdz; }
        } catch(std::exception& e) {
#pragma omp critical
            err = e.what();
        }
    }
    if(!err.empty()) { g_error = err; return -1; }
    return 0;
}

/// potential + gradient in cylindrical coordinates (R,z,phi) -> (Phi, dR, dz, dphi) and Hessian
int ref_eval_cyl_many(void* handle, long n, const double* pos, double* phi, double* grad, double* hess) {
    const potential::BasePotential& pot = *static_cast<PotHandle*>(handle)->pot;
    try {
        for(long i = 0; i < n; i++) {
            double p; coord::GradCyl g; coord::HessCyl h;
            pot.eval(coord::PosCyl(pos[3*i], pos[3*i+1], pos[3*i+2]), &p, grad ? &g : NULL, hess ? &h : NULL);
            if(phi) phi[i] = p;
            if(grad) { grad[3*i] = g.dR; grad[3*i+1] = g.dz; grad[3*i+2] = g.dphi; }
            if(hess) { hess[6*i] = h.dR2; hess[6*i+1] = h.dz2; hess[6*i+2] = h.dphi2;
                       hess[6*i+3] = h.dRdz; hess[6*i+4] = h.dzdphi; hess[6*i+5] = h.dRdphi; }
        }
    } catch(std::exception& e) { g_error = e.what(); return -1; }
    return 0;
}

/// integrate n orbits with DOP853 (accuracy acc) for times T[i] in a frame rotating with Omega;
/// output the final phase-space point, the number of accepted steps and a status
/// (0 = reached T, 1 = stopped early: zero/non-finite step or maxSteps)
int ref_orbits_many(void* handle, long n, const double* ic, const double* T, double Omega,
    double accuracy, long maxSteps, double* final, long* nsteps, int* status, int nthreads)
{
    const potential::BasePotential& pot = *static_cast<PotHandle*>(handle)->pot;
    setThreads(nthreads);
    orbit::OrbitIntParams params(accuracy, maxSteps > 0 ? (size_t)maxSteps : (size_t)1e8);
    std::string err;
#pragma omp parallel for schedule(dynamic, 1)
    for(long i = 0; i < n; i++) {
        try {
            long cnt = 0;
            orbit::Trajectory traj;
            orbit::OrbitIntegrator<coord::Car> orbint(pot, Omega, params);
            orbint.addRuntimeFnc(orbit::PtrRuntimeFnc(new StepCounter(orbint, &cnt)));
            // final point recorded as the reference's Python orbit() does: a runtime trajectory
            // with an infinite sampling interval (interface_python.cpp:8126-8127, orbit.cpp:19-25)
            orbint.addRuntimeFnc(orbit::PtrRuntimeFnc(new orbit::RuntimeTrajectory(orbint, INFINITY, traj)));
            coord::PosVelCar ic6(ic + 6*i);
            orbint.init(ic6);
            orbint.run(T[i]);
            if(traj.empty()) ic6.unpack_to(final + 6*i);
            else traj[0].first.unpack_to(final + 6*i);
            // the reference reports no status: infer "stopped before T" from the last recorded time
            const bool reachedEnd = T[i] == 0 || (!traj.empty() && traj[0].second == T[i]);
            if(nsteps) nsteps[i] = cnt;
            if(status) status[i] = reachedEnd ? 0 : 1;
        } catch(std::exception& e) {
            if(status) status[i] = -1;
#pragma omp critical
            err = e.what();
        }
    }
    if(!err.empty()) { g_error = err; return -1; }
    return 0;
}

/// trajectories sampled at trajSize regular times 0, T/(trajSize-1), ..., T (the reference's
/// RuntimeTrajectory with samplingInterval = T/(trajSize-1), as its Python orbit(trajsize=...));
/// traj: n x trajSize x 6, NaN where the orbit produced no sample
int ref_orbits_traj_many(void* handle, long n, const double* ic, const double* T, double Omega,
    double accuracy, long maxSteps, int trajSize, double* traj, int nthreads)
{
    const potential::BasePotential& pot = *static_cast<PotHandle*>(handle)->pot;
    setThreads(nthreads);
    orbit::OrbitIntParams params(accuracy, maxSteps > 0 ? (size_t)maxSteps : (size_t)1e8);
    std::string err;
#pragma omp parallel for schedule(dynamic, 1)
    for(long i = 0; i < n; i++) {
        try {
            for(long k = 0; k < (long)trajSize * 6; k++) traj[i * trajSize * 6 + k] = NAN;
            orbit::Trajectory tr;
            orbit::OrbitIntegrator<coord::Car> orbint(pot, Omega, params);
            orbint.addRuntimeFnc(orbit::PtrRuntimeFnc(
                new orbit::RuntimeTrajectory(orbint, fabs(T[i]) / (trajSize - 1), tr)));
            orbint.init(coord::PosVelCar(ic + 6*i));
            orbint.run(T[i]);
            for(size_t k = 0; k < tr.size() && (long)k < trajSize; k++)
                tr[k].first.unpack_to(traj + (i * trajSize + k) * 6);
        } catch(std::exception& e) {
#pragma omp critical
            err = e.what();
        }
    }
    if(!err.empty()) { g_error = err; return -1; }
    return 0;
}

/// the number of potential evaluations each orbit of ref_orbits_many costs (counting wrapper)
int ref_orbits_evals(void* handle, long n, const double* ic, const double* T, double Omega,
    double accuracy, long maxSteps, long long* nevals, int nthreads)
{
    potential::PtrPotential base = static_cast<PotHandle*>(handle)->pot;
    setThreads(nthreads);
    orbit::OrbitIntParams params(accuracy, maxSteps > 0 ? (size_t)maxSteps : (size_t)1e8);
    std::string err;
#pragma omp parallel for schedule(dynamic, 1)
    for(long i = 0; i < n; i++) {
        try {
            CountingPotential cnt(base);
            orbit::OrbitIntegrator<coord::Car> orbint(cnt, Omega, params);
            orbint.init(coord::PosVelCar(ic + 6*i));
            orbint.run(T[i]);
            nevals[i] = cnt.count;
        } catch(std::exception& e) {
#pragma omp critical
            err = e.what();
        }
    }
    if(!err.empty()) { g_error = err; return -1; }
    return 0;
}

/// Staeckel-fudge actions with a given focal distance per point (Cartesian posvel input);
/// if countEvals is not NULL, it receives the number of potential evaluations per point
int ref_actions_fd_many(void* handle, long n, const double* posvel, const double* fd, double* act,
    long long* countEvals, int nthreads)
{
    potential::PtrPotential base = static_cast<PotHandle*>(handle)->pot;
    setThreads(nthreads);
    std::string err;
#pragma omp parallel for schedule(dynamic, 64)
    for(long i = 0; i < n; i++) {
        try {
            CountingPotential cnt(base);
            actions::Actions a;
            actions::evalAxisymFudge(cnt, coord::toPosVelCyl(coord::PosVelCar(posvel + 6*i)), &a, NULL, NULL, fd[i]);
            act[3*i] = a.Jr; act[3*i+1] = a.Jz; act[3*i+2] = a.Jphi;
            if(countEvals) countEvals[i] = cnt.count;
        } catch(std::exception& e) {
#pragma omp critical
            err = e.what();
        }
    }
    if(!err.empty()) { g_error = err; return -1; }
    return 0;
}

/// Staeckel-fudge actions, angles and frequencies with a given focal distance (f1 outputs)
int ref_actions_angles_fd_many(void* handle, long n, const double* posvel, const double* fd,
    double* act, double* ang, double* freq, int nthreads)
{
    potential::PtrPotential base = static_cast<PotHandle*>(handle)->pot;
    setThreads(nthreads);
    std::string err;
#pragma omp parallel for schedule(dynamic, 64)
    for(long i = 0; i < n; i++) {
        try {
            actions::Actions a; actions::Angles t; actions::Frequencies f;
            actions::evalAxisymFudge(*base, coord::toPosVelCyl(coord::PosVelCar(posvel + 6*i)),
                act ? &a : NULL, ang ? &t : NULL, freq ? &f : NULL, fd[i]);
            if(act)  { act[3*i] = a.Jr; act[3*i+1] = a.Jz; act[3*i+2] = a.Jphi; }
            if(ang)  { ang[3*i] = t.thetar; ang[3*i+1] = t.thetaz; ang[3*i+2] = t.thetaphi; }
            if(freq) { freq[3*i] = f.Omegar; freq[3*i+1] = f.Omegaz; freq[3*i+2] = f.Omegaphi; }
        } catch(std::exception& e) {
#pragma omp critical
            err = e.what();
        }
    }
    if(!err.empty()) { g_error = err; return -1; }
    return 0;
}

void* ref_actionfinder_create(void* handle) {
    try {
        AfHandle* h = new AfHandle;
        h->cnt.reset(new CountingPotential(static_cast<PotHandle*>(handle)->pot));
        h->af.reset(new actions::ActionFinderAxisymFudge(h->cnt, false));
        h->cnt->count = 0;
        return h;
    } catch(std::exception& e) { g_error = e.what(); return NULL; }
}

void ref_actionfinder_free(void* af) { delete static_cast<AfHandle*>(af); }

/// total number of potential evaluations made through the action finder since creation / reset
long long ref_actionfinder_evalcount(void* af, int reset) {
    AfHandle* h = static_cast<AfHandle*>(af);
    long long c = h->cnt->count;
    if(reset) h->cnt->count = 0;
    return c;
}

int ref_actionfinder_many(void* handle, long n, const double* posvel, double* act, double* fdOut, int nthreads) {
    const actions::ActionFinderAxisymFudge& af = *static_cast<AfHandle*>(handle)->af;
    setThreads(nthreads);
    std::string err;
#pragma omp parallel for schedule(dynamic, 64)
    for(long i = 0; i < n; i++) {
        try {
            coord::PosVelCyl p = coord::toPosVelCyl(coord::PosVelCar(posvel + 6*i));
            actions::Actions a;
            af.eval(p, &a);
            act[3*i] = a.Jr; act[3*i+1] = a.Jz; act[3*i+2] = a.Jphi;
            if(fdOut) fdOut[i] = af.focalDistance(p);
        } catch(std::exception& e) {
#pragma omp critical
            err = e.what();
        }
    }
    if(!err.empty()) { g_error = err; return -1; }
    return 0;
}

/// sizes of the action finder's tables: [sizeE, sizeL, nLofE, nRofL, nPhiofR]
int ref_actionfinder_table_sizes(void* handle, long* sizes) {
    const actions::ActionFinderAxisymFudge& af = *static_cast<AfHandle*>(handle)->af;
    sizes[0] = af.interpD.xval.size();
    sizes[1] = af.interpD.yval.size();
    sizes[2] = af.interp.LofE.xval.size();
    sizes[3] = af.interp.RofL.xval.size();
    sizes[4] = af.interp.PhiofR.xval.size();
    return 0;
}

/// copy the focal-distance table (grids in scaled E and scaled Lz/Lcirc, values sizeE x sizeL)
/// and the Interpolator's LofE / RofL / PhiofR quintic splines (x, f, f', f'') plus scalars
/// [invPhi0(finder), invPhi0(interp), slopeOut, coefOut, massOut]
int ref_actionfinder_tables(void* handle, double* gridE, double* gridL, double* delta,
    double* lofe, double* rofl, double* phiofr, double* scalars)
{
    const actions::ActionFinderAxisymFudge& af = *static_cast<AfHandle*>(handle)->af;
    std::copy(af.interpD.xval.begin(), af.interpD.xval.end(), gridE);
    std::copy(af.interpD.yval.begin(), af.interpD.yval.end(), gridL);
    std::copy(af.interpD.fval.begin(), af.interpD.fval.end(), delta);
    const math::QuinticSpline* spl[3] = { &af.interp.LofE, &af.interp.RofL, &af.interp.PhiofR };
    double* out[3] = { lofe, rofl, phiofr };
    for(int s = 0; s < 3; s++) {
        size_t m = spl[s]->xval.size();
        std::copy(spl[s]->xval.begin(),  spl[s]->xval.end(),  out[s]);
        std::copy(spl[s]->fval.begin(),  spl[s]->fval.end(),  out[s] + m);
        std::copy(spl[s]->fder.begin(),  spl[s]->fder.end(),  out[s] + 2*m);
        std::copy(spl[s]->fder2.begin(), spl[s]->fder2.end(), out[s] + 3*m);
    }
    scalars[0] = af.invPhi0;
    scalars[1] = af.interp.invPhi0;
    scalars[2] = af.interp.slopeOut;
    scalars[3] = af.interp.coefOut;
    scalars[4] = af.interp.massOut;
    return 0;
}

/// L_circ(E) through the reference Interpolator of the action finder
int ref_actionfinder_lcirc(void* handle, long n, const double* E, double* L) {
    const actions::ActionFinderAxisymFudge& af = *static_cast<AfHandle*>(handle)->af;
    for(long i = 0; i < n; i++) L[i] = af.interp.L_circ(E[i]);
    return 0;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// The reference's root finder on a test function (checker of the engine's restatement)

namespace {
/// sum_k c[k] x^k and its derivative by Horner's rule: a test function with one derivative
class PolyFnc : public math::IFunction {
    const double* c;
    int n;
public:
    PolyFnc(const double* c_, int n_) : c(c_), n(n_) {}
    virtual void evalDeriv(const double x, double* val, double* der, double*) const {
        double v = 0, d = 0;
        for(int k = n - 1; k >= 0; k--) { d = d * x + v; v = v * x + c[k]; }
        if(val) *val = v;
        if(der) *der = d;
    }
    virtual unsigned int numDerivs() const { return 1; }
};
}  // namespace

extern "C" {
/// math::findRoot (src/math_core.cpp:895-1041) of the polynomial c[0..n-1] on [lo, hi]
int ref_find_root_poly(const double* c, int n, double lo, double hi, double reltol, double* root)
{
    try { *root = math::findRoot(PolyFnc(c, n), lo, hi, reltol); return 0; }
    catch(std::exception& e) { g_error = e.what(); return -1; }
}
}  // extern "C"

// ------------------------------------------------------------------------------------------
// The reference's Legendre, multiple-angle and interval-scaling routines (checkers of the
// engine's restatements)

extern "C" {
/// math::sphHarmArray (src/math_sphharm.cpp:63-132): lmax-m+1 values and derivatives
int ref_sph_harm_array(int lmax, int m, double tau, double* P, double* dP, double* d2P)
{
    try { math::sphHarmArray(lmax, m, tau, P, dP, d2P); return 0; }
    catch(std::exception& e) { g_error = e.what(); return -1; }
}

/// math::trigMultiAngle (src/math_sphharm.cpp:134-154)
int ref_trig_multi_angle(double phi, int m, int needSine, double* out)
{
    math::trigMultiAngle(phi, m, needSine != 0, out);
    return 0;
}

/// math::unscale / math::scale (src/math_core.cpp:296-396) of kind 0 ScalingInf, 1 ScalingSemiInf(a),
/// 2 ScalingCub(a, b)
int ref_unscale(int kind, double a, double b, double s, double* u, double* duds)
{
    if(kind == 0) *u = math::unscale(math::ScalingInf(), s, duds);
    else if(kind == 1) *u = math::unscale(math::ScalingSemiInf(a), s, duds);
    else *u = math::unscale(math::ScalingCub(a, b), s, duds);
    return 0;
}
int ref_scale(int kind, double a, double b, double u, double* s)
{
    if(kind == 0) *s = math::scale(math::ScalingInf(), u);
    else if(kind == 1) *s = math::scale(math::ScalingSemiInf(a), u);
    else *s = math::scale(math::ScalingCub(a, b), u);
    return 0;
}
}  // extern "C"

// ------------------------------------------------------------------------------------------
// The reference's Poisson solve (checker of the engine's Multipole construction from densities)

namespace potential {
// defined with external linkage in src/potential_multipole.cpp:1013-1114 (not in its header)
void computePotentialCoefsFromSource(const BaseDensity& dens, const math::SphHarmIndices& ind,
    const std::vector<double>& gridRadii, std::vector< std::vector<double> > coefs[2]);
}

extern "C" {
/// Multipole::create (src/potential_multipole.cpp:1400-1441) from the sum of the densities given
/// as key=value strings (createDensity, src/potential_factory.h:31-33) with the Multipole's
/// parameters (lmax, mmax, gridSizeR, rmin, rmax, symmetry, fixOrder): its coefficients at full
/// precision (getCoefs).  Call with radii == NULL for the sizes.
int ref_multipole_from_density(const char* multipoleParams, int ncomp, const char* const* densityParams,
    int* nr, int* nc, double* radii, double* Phi, double* dPhi)
{
    try {
        std::vector<potential::PtrDensity> comps;
        for(int k = 0; k < ncomp; k++)
            comps.push_back(potential::createDensity(utils::KeyValueMap(std::string(densityParams[k]))));
        potential::PtrDensity dens = ncomp == 1 ? comps[0] :
            potential::PtrDensity(new potential::CompositeDensity(comps));
        utils::KeyValueMap mp{std::string(multipoleParams)};
        const int lmax = mp.getInt("lmax", 6);
        std::shared_ptr<const potential::Multipole> mul = potential::Multipole::create(*dens,
            potential::getSymmetryTypeByName(mp.getString("symmetry")), lmax, mp.getInt("mmax", lmax),
            mp.getInt("gridSizeR", 25), mp.getDouble("rmin", 0), mp.getDouble("rmax", 0), mp.getBool("fixOrder", false));
        std::vector<double> r;
        std::vector<std::vector<double> > P, D;
        mul->getCoefs(r, P, D);
        if(mp.getBool("raw", false)) {
            // the coefficients of the Poisson solve itself on the same grid (getCoefs returns the
            // values re-derived from the spline interpolator), with the source's angular order
            // (createMultipole, src/potential_multipole.cpp:1418-1432), restricted to the output terms
            const coord::SymmetryType symSrc = dens->symmetry();
            int lmaxSrc = std::max<int>(lmax + 6, 12), mmaxSrc = std::max<int>(mp.getInt("mmax", lmax) + 6, 12);
            if(mp.getBool("fixOrder", false)) { lmaxSrc = lmax; mmaxSrc = mp.getInt("mmax", lmax); }
            if(isSpherical(symSrc)) lmaxSrc = 0;
            if(isZRotSymmetric(symSrc)) mmaxSrc = 0;
            std::vector<std::vector<double> > coefs[2];
            potential::computePotentialCoefsFromSource(*dens, math::SphHarmIndices(lmaxSrc, mmaxSrc, symSrc), r, coefs);
            for(size_t c = 0; c < P.size(); c++) {
                const bool nonzero = !(math::allZeros(P[c]) && math::allZeros(D[c]));
                P[c] = nonzero && c < coefs[0].size() ? coefs[0][c] : std::vector<double>(r.size(), 0.);
                D[c] = nonzero && c < coefs[1].size() ? coefs[1][c] : std::vector<double>(r.size(), 0.);
            }
        }
        if(radii) {
            for(size_t k = 0; k < r.size(); k++) radii[k] = r[k];
            for(size_t c = 0; c < P.size(); c++)
                for(size_t k = 0; k < r.size(); k++) {
                    Phi[c * r.size() + k] = P[c][k];
                    dPhi[c * r.size() + k] = D[c][k];
                }
        }
        *nr = static_cast<int>(r.size());
        *nc = static_cast<int>(P.size());
        return 0;
    } catch(std::exception& e) { g_error = e.what(); return -1; }
}

/// the reference's Multipole from the sum of densities, as a potential handle (in memory: its
/// tables come from the Poisson solve itself, not from a coefficient file)
void* ref_multipole_potential_from_density(const char* multipoleParams, int ncomp, const char* const* densityParams)
{
    try {
        std::vector<potential::PtrDensity> comps;
        for(int k = 0; k < ncomp; k++)
            comps.push_back(potential::createDensity(utils::KeyValueMap(std::string(densityParams[k]))));
        potential::PtrDensity dens = ncomp == 1 ? comps[0] :
            potential::PtrDensity(new potential::CompositeDensity(comps));
        utils::KeyValueMap mp{std::string(multipoleParams)};
        const int lmax = mp.getInt("lmax", 6);
        PotHandle* h = new PotHandle;
        h->pot = potential::Multipole::create(*dens, potential::getSymmetryTypeByName(mp.getString("symmetry")), lmax,
            mp.getInt("mmax", lmax), mp.getInt("gridSizeR", 25), mp.getDouble("rmin", 0), mp.getDouble("rmax", 0),
            mp.getBool("fixOrder", false));
        return h;
    } catch(std::exception& e) { g_error = e.what(); return NULL; }
}
}  // extern "C"
