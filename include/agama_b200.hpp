/* C++ mirror of the reference's API for the Multipole / orbit / Staeckel-fudge path, header-only,
   over the C-ABI of agama_b200.h.  Names, argument meaning and error behaviour follow the
   reference's C++ classes so that C++ callers switch by changing the namespace:

     coord::PosCar, PosCyl, PosVelCar, PosVelCyl, GradCar, HessCar      src/coord.h:190-501
     potential::Multipole::eval / value / density                        src/potential_base.h:153-164
       (BasePotential::eval: null output pointers mean "not requested")
     potential::R_circ, R_from_Lz, R_max, findPlanarOrbitExtent          src/potential_utils.cpp:617-729
     actions::Actions, Angles, Frequencies                               src/actions_base.h:14-45
     actions::ActionFinderAxisymFudge::eval / actions                    src/actions_base.h:65-75,
                                                                         src/actions_staeckel.cpp:954-979
     orbit::OrbitIntParams, orbit::integrate (final point of a DOP853     src/orbit.h:116-129, 165-315
       orbit in the frame rotating with Omega), orbit::integrateTraj        src/orbit.h:297-316

   Errors raise std::runtime_error with the engine's message, as the reference's constructors and
   factories throw; evaluations of points without a value (unbound orbits) give NaN as there, and
   the radius routines return NaN on failure as the plain-C interface does.
   The batched members (evalmany..., integratemany) take whole arrays in one call; the reference
   batches the same operations only in its Python binding. */
#ifndef AGAMA_B200_HPP
#define AGAMA_B200_HPP

#include "agama_b200.h"
#include <cmath>
#include <cstddef>
#include <memory>
#include <stdexcept>
#include <algorithm>
#include <string>
#include <utility>
#include <vector>

namespace agama_b200 {

namespace detail {
inline void check(int rc) { if(rc != 0) throw std::runtime_error(agama_getError()); }
}

namespace coord {
struct PosCar { double x, y, z; PosCar() : x(0), y(0), z(0) {} PosCar(double x_, double y_, double z_) : x(x_), y(y_), z(z_) {} };
struct PosCyl { double R, z, phi; PosCyl() : R(0), z(0), phi(0) {} PosCyl(double R_, double z_, double p_) : R(R_), z(z_), phi(p_) {} };
struct VelCar { double vx, vy, vz; VelCar() : vx(0), vy(0), vz(0) {} VelCar(double a, double b, double c) : vx(a), vy(b), vz(c) {} };
struct VelCyl { double vR, vz, vphi; VelCyl() : vR(0), vz(0), vphi(0) {} VelCyl(double a, double b, double c) : vR(a), vz(b), vphi(c) {} };
struct PosVelCar : PosCar, VelCar {
    PosVelCar() {}
    PosVelCar(double x_, double y_, double z_, double vx_, double vy_, double vz_) : PosCar(x_, y_, z_), VelCar(vx_, vy_, vz_) {}
};
struct PosVelCyl : PosCyl, VelCyl {
    PosVelCyl() {}
    PosVelCyl(double R_, double z_, double p_, double vR_, double vz_, double vphi_) : PosCyl(R_, z_, p_), VelCyl(vR_, vz_, vphi_) {}
};
struct GradCar { double dx, dy, dz; };
struct HessCar { double dx2, dy2, dz2, dxdy, dydz, dxdz; };

/// cylindrical -> Cartesian phase-space point (coord::toPosVelCar)
inline PosVelCar toPosVelCar(const PosVelCyl& p)
{
    const double c = std::cos(p.phi), s = std::sin(p.phi);
    return PosVelCar(p.R * c, p.R * s, p.z, p.vR * c - p.vphi * s, p.vR * s + p.vphi * c, p.vz);
}
}  // namespace coord

namespace potential {

/** A Multipole potential resident on the current CUDA device, read from the reference's
    coefficient file (the potential::Multipole that createPotential makes of it). */
class Multipole {
    std::shared_ptr<agama_Potential> h;
public:
    explicit Multipole(const std::string& coefFile)
    {
        agama_Potential* p = agama_createPotential(("type=Multipole, file=" + coefFile).c_str());
        if(!p) throw std::runtime_error(agama_getError());
        h.reset(p, agama_deletePotential);
    }
    /// from the spherical-harmonic coefficients at the radial grid: Phi[c][k], dPhi[c][k] for the
    /// coefficient index c = l (l + 1) + m and radius k (Multipole(radii, Phi, dPhi),
    /// src/potential_multipole.h:257-266)
    Multipole(const std::vector<double>& radii, const std::vector<std::vector<double> >& Phi,
        const std::vector<std::vector<double> >& dPhi)
    {
        const size_t nr = radii.size(), nc = Phi.size();
        if(dPhi.size() != nc) throw std::invalid_argument("Multipole: Phi and dPhi differ in size");
        std::vector<double> P(nc * nr), D(nc * nr);
        for(size_t c = 0; c < nc; c++) {
            if(Phi[c].size() != nr || dPhi[c].size() != nr)
                throw std::invalid_argument("Multipole: each coefficient needs one value per radius");
            std::copy(Phi[c].begin(), Phi[c].end(), P.begin() + c * nr);
            std::copy(dPhi[c].begin(), dPhi[c].end(), D.begin() + c * nr);
        }
        agama_Potential* p = agama_createMultipoleFromCoefs(static_cast<int>(nr), radii.data(), static_cast<int>(nc),
            P.data(), D.data());
        if(!p) throw std::runtime_error(agama_getError());
        h.reset(p, agama_deletePotential);
    }
    const agama_Potential* handle() const { return h.get(); }
    std::string name() const { return "Multipole"; }

    /// BasePotential::eval in Cartesian coordinates; the time is ignored (a static potential)
    void eval(const coord::PosCar& pos, double* potential, coord::GradCar* deriv = NULL,
        coord::HessCar* deriv2 = NULL, double time = 0) const
    {
        const double x[3] = { pos.x, pos.y, pos.z };
        double g[3], hs[6], phi = NAN;
        detail::check(agama_evalPotentialMany(h.get(), 1, x, time, &phi, deriv ? g : NULL, deriv2 ? hs : NULL));
        if(potential) *potential = phi;
        if(deriv) { deriv->dx = g[0]; deriv->dy = g[1]; deriv->dz = g[2]; }
        if(deriv2) {    // the engine's order xx, yy, zz, xy, yz, zx
            deriv2->dx2 = hs[0]; deriv2->dy2 = hs[1]; deriv2->dz2 = hs[2];
            deriv2->dxdy = hs[3]; deriv2->dydz = hs[4]; deriv2->dxdz = hs[5];
        }
    }
    double value(const coord::PosCar& pos, double time = 0) const { double p; eval(pos, &p, NULL, NULL, time); return p; }

    /// density (Laplacian / 4 pi), BaseDensity::density
    double density(const coord::PosCar& pos, double time = 0) const
    {
        const double x[3] = { pos.x, pos.y, pos.z };
        double rho = NAN;
        detail::check(agama_evalDensityMany(h.get(), 1, x, time, &rho));
        return rho;
    }

    /// n points in one call: potential, gradient and Hessian (any output may be NULL)
    void evalmanyCar(size_t n, const coord::PosCar* pos, double* potential, coord::GradCar* deriv = NULL,
        coord::HessCar* deriv2 = NULL) const
    {
        std::vector<double> x(3 * n), g(deriv ? 3 * n : 0), hs(deriv2 ? 6 * n : 0), phi(n);
        for(size_t i = 0; i < n; i++) { x[3 * i] = pos[i].x; x[3 * i + 1] = pos[i].y; x[3 * i + 2] = pos[i].z; }
        detail::check(agama_evalPotentialMany(h.get(), static_cast<long>(n), x.data(), 0, phi.data(),
            deriv ? g.data() : NULL, deriv2 ? hs.data() : NULL));
        for(size_t i = 0; i < n; i++) {
            if(potential) potential[i] = phi[i];
            if(deriv) { deriv[i].dx = g[3 * i]; deriv[i].dy = g[3 * i + 1]; deriv[i].dz = g[3 * i + 2]; }
            if(deriv2) {
                const double* q = &hs[6 * i];
                deriv2[i].dx2 = q[0]; deriv2[i].dy2 = q[1]; deriv2[i].dz2 = q[2];
                deriv2[i].dxdy = q[3]; deriv2[i].dydz = q[4]; deriv2[i].dxdz = q[5];
            }
        }
    }
};

typedef std::shared_ptr<const Multipole> PtrPotential;

inline double R_circ(const Multipole& pot, double E) { return agama_R_circ(pot.handle(), E); }
inline double R_from_Lz(const Multipole& pot, double Lz) { return agama_R_from_Lz(pot.handle(), Lz); }
inline double R_max(const Multipole& pot, double E) { return agama_R_max(pot.handle(), E); }
inline void findPlanarOrbitExtent(const Multipole& pot, double E, double L, double& R1, double& R2)
{
    agama_findPlanarOrbitExtent(pot.handle(), E, L, &R1, &R2);
}

}  // namespace potential

namespace actions {

struct Actions { double Jr, Jz, Jphi; Actions() : Jr(0), Jz(0), Jphi(0) {} Actions(double a, double b, double c) : Jr(a), Jz(b), Jphi(c) {} };
struct Angles { double thetar, thetaz, thetaphi; Angles() : thetar(0), thetaz(0), thetaphi(0) {} };
struct Frequencies { double Omegar, Omegaz, Omegaphi; Frequencies() : Omegar(0), Omegaz(0), Omegaphi(0) {} };

/** ActionFinderAxisymFudge: the Staeckel fudge with the focal distance from the finder's own table
    (built on the device from shell orbits, as the reference's constructor builds it). */
class ActionFinderAxisymFudge {
    potential::PtrPotential pot;
    std::shared_ptr<agama_ActionFinder> h;
public:
    explicit ActionFinderAxisymFudge(const potential::PtrPotential& potential) : pot(potential)
    {
        if(!pot) throw std::invalid_argument("ActionFinderAxisymFudge: null potential");
        agama_ActionFinder* a = agama_createActionFinder(pot->handle());
        if(!a) throw std::runtime_error(agama_getError());
        h.reset(a, agama_deleteActionFinder);
    }
    std::string name() const { return "AxisymFudge"; }

    /// BaseActionFinder::eval: any of the outputs may be NULL
    void eval(const coord::PosVelCyl& point, Actions* act, Angles* ang = NULL, Frequencies* freq = NULL) const
    {
        const coord::PosVelCar c = coord::toPosVelCar(point);
        const double pv[6] = { c.x, c.y, c.z, c.vx, c.vy, c.vz };
        double a[3], t[3], f[3];
        if(act || ang || freq)
            detail::check(agama_evalActionsAnglesFrequenciesMany(h.get(), 1, pv, a, ang ? t : NULL, freq ? f : NULL));
        if(act) *act = Actions(a[0], a[1], a[2]);
        if(ang) { ang->thetar = t[0]; ang->thetaz = t[1]; ang->thetaphi = t[2]; }
        if(freq) { freq->Omegar = f[0]; freq->Omegaz = f[1]; freq->Omegaphi = f[2]; }
    }
    Actions actions(const coord::PosVelCyl& point) const { Actions a; eval(point, &a); return a; }

    /// the actions of n Cartesian points in one call
    void evalmany(size_t n, const coord::PosVelCar* points, Actions* act) const
    {
        std::vector<double> pv(6 * n), a(3 * n);
        for(size_t i = 0; i < n; i++) {
            const coord::PosVelCar& p = points[i];
            double* q = &pv[6 * i];
            q[0] = p.x; q[1] = p.y; q[2] = p.z; q[3] = p.vx; q[4] = p.vy; q[5] = p.vz;
        }
        detail::check(agama_evalActionsMany(h.get(), static_cast<long>(n), pv.data(), a.data(), NULL));
        for(size_t i = 0; i < n; i++) act[i] = Actions(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
    }
};

}  // namespace actions

namespace orbit {

/// accuracy and step limit of the DOP853 integrator (OrbitIntParams, src/orbit.h:116-129)
struct OrbitIntParams {
    double accuracy;
    size_t maxNumSteps;
    explicit OrbitIntParams(double acc = 1e-8, size_t maxSteps = 100000000) : accuracy(acc), maxNumSteps(maxSteps) {}
};

/** n orbits from ic[i] for times T[i] in the frame rotating with Omega about z: final points,
    and optionally accepted step counts and statuses (0 ok, 1 step limit, 2 zero / non-finite
    step, 3 non-finite error estimate). */
inline void integratemany(size_t n, const coord::PosVelCar* ic, const double* T, const potential::Multipole& pot,
    double Omega, const OrbitIntParams& params, coord::PosVelCar* finalPoints, long* numSteps = NULL,
    int* status = NULL)
{
    std::vector<double> in(6 * n), out(6 * n);
    std::vector<long> steps(n);
    std::vector<int> st(n);
    for(size_t i = 0; i < n; i++) {
        double* q = &in[6 * i];
        q[0] = ic[i].x; q[1] = ic[i].y; q[2] = ic[i].z; q[3] = ic[i].vx; q[4] = ic[i].vy; q[5] = ic[i].vz;
    }
    detail::check(agama_integrateOrbitsMany(pot.handle(), static_cast<long>(n), in.data(), T, Omega, params.accuracy,
        static_cast<long>(params.maxNumSteps), out.data(), steps.data(), st.data()));
    for(size_t i = 0; i < n; i++) {
        const double* q = &out[6 * i];
        finalPoints[i] = coord::PosVelCar(q[0], q[1], q[2], q[3], q[4], q[5]);
        if(numSteps) numSteps[i] = steps[i];
        if(status) status[i] = st[i];
    }
}

/// one orbit: its final point (orbit::integrateTraj with a final-point trajectory)
inline coord::PosVelCar integrate(const coord::PosVelCar& ic, double T, const potential::Multipole& pot,
    double Omega = 0, const OrbitIntParams& params = OrbitIntParams())
{
    coord::PosVelCar out;
    integratemany(1, &ic, &T, pot, Omega, params, &out);
    return out;
}

/// points of a trajectory with their times (orbit::Trajectory, src/orbit.h:82)
typedef std::vector<std::pair<coord::PosVelCar, double> > Trajectory;

/** The trajectory of one orbit sampled every samplingInterval from startTime to startTime +
    totalTime (orbit::integrateTraj, src/orbit.h:297-316, with the reference's RuntimeTrajectory:
    7th-order dense output of the DOP853 steps).  The engine samples at regular times that end on
    totalTime, so samplingInterval must divide totalTime (to 1e-12 relative); recording every step
    (samplingInterval = 0) is not offered. */
inline Trajectory integrateTraj(const coord::PosVelCar& initialConditions, double totalTime, double samplingInterval,
    const potential::Multipole& pot, double Omega = 0, const OrbitIntParams& params = OrbitIntParams(),
    double startTime = 0)
{
    if(!(samplingInterval > 0))
        throw std::invalid_argument("integrateTraj: the engine samples at regular intervals (samplingInterval > 0)");
    const double steps = std::fabs(totalTime) / samplingInterval;
    const double k = std::floor(steps + 0.5);
    if(std::fabs(steps - k) > 1e-12 * std::fmax(1.0, steps))
        throw std::invalid_argument("integrateTraj: samplingInterval must divide totalTime");
    const int trajSize = static_cast<int>(k) + 1;
    const double ic[6] = { initialConditions.x, initialConditions.y, initialConditions.z,
                           initialConditions.vx, initialConditions.vy, initialConditions.vz };
    std::vector<double> traj(6 * static_cast<size_t>(std::max(trajSize, 2)));
    long numSteps = 0;
    int status = 0;
    detail::check(agama_integrateOrbitsTrajectoryMany(pot.handle(), 1, ic, &totalTime, Omega, params.accuracy,
        static_cast<long>(params.maxNumSteps), std::max(trajSize, 2), traj.data(), NULL, &numSteps, &status));
    Trajectory out;
    for(int j = 0; j < trajSize; j++) {
        const double* q = &traj[6 * j];
        if(!std::isfinite(q[0])) break;           // the orbit stopped before this sample
        const double t = trajSize > 1 ? totalTime * j / (trajSize - 1) : 0;
        out.push_back(std::make_pair(coord::PosVelCar(q[0], q[1], q[2], q[3], q[4], q[5]), startTime + t));
    }
    return out;
}

}  // namespace orbit

}  // namespace agama_b200

#endif  // AGAMA_B200_HPP
