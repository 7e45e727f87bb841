/* Drop-in classes for C++ code built against the reference library (Agama): the engine's
   potential and action finder as subclasses of the reference's own abstract interfaces, so that
   reference code holding a potential::PtrPotential or an actions::PtrActionFinder runs on the
   B200 engine without other changes.  Header-only over the C-ABI of agama_b200.h; include it
   after putting the reference's src/ directory on the include path:

     agama_b200::MultipoleB200 : potential::BasePotentialCyl      src/potential_base.h:237-262
       eval(PosCar / PosCyl / PosSph, Phi*, Grad*, Hess*, t)    src/potential_base.h:153-164
         (through the reference's non-virtual front-ends; the Cartesian and cylindrical forms are
         one engine call each, the spherical form converts through the reference's
         coord::evalAndConvert as BasePotentialCyl does)
       symmetry(), name() = "Multipole"                          src/potential_multipole.h:283-284
       evalmanyDensityCar / Cyl (virtual in BaseDensity)         src/potential_base.h:87-99
         -> one batched device call for the whole array
       evalmanyCar / evalmanyCyl: potential, gradient, Hessian of whole arrays in one call, in
         the house style of evalmanyDensityCar (the reference has no batched potential method)
     agama_b200::ActionFinderB200 : actions::BaseActionFinder     src/actions_base.h:49-82
       eval(PosVelCyl, Actions*, Angles*, Frequencies*)          src/actions_staeckel.cpp:954-979
       name() as ActionFinderAxisymFudge::name                    src/actions_staeckel.cpp:1031-1035
       evalmany(n, points, act, ang, freq): whole arrays in one call

   Semantics follow the reference classes: null output pointers mean "not requested", unbound
   points give NaN actions, construction failures throw std::runtime_error with the engine's
   message.  Every single-point call is one kernel launch and a synchronisation (tens of
   microseconds): code that evaluates many points should use the evalmany members. */
#ifndef AGAMA_B200_REFERENCE_HPP
#define AGAMA_B200_REFERENCE_HPP

#include "agama_b200.h"
#include "potential_base.h"
#include "actions_base.h"
#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace agama_b200 {

namespace detail {
inline void checkRef(int rc) { if(rc != 0) throw std::runtime_error(agama_getError()); }
}  // namespace detail

/** A Multipole potential evaluated on the B200 engine, usable wherever the reference takes a
    potential::BasePotential (for example a potential::PtrPotential given to the reference's own
    action finders, orbit integrators or radius routines). */
class MultipoleB200 : public potential::BasePotentialCyl {
public:
    /// from a Multipole coefficient file written by the reference (writePotential)
    explicit MultipoleB200(const std::string& coefFile)
        : h(agama_createPotential(("file=" + coefFile).c_str()))
    {
        if(!h) throw std::runtime_error(agama_getError());
        readInfo();
    }
    /// from coefficient arrays, as the reference's Multipole(gridRadii, Phi, dPhi) constructor
    /// (src/potential_multipole.h:235-243): Phi[c][k], dPhi[c][k] for c = l(l+1)+m, k = radius
    MultipoleB200(const std::vector<double>& radii, const std::vector<std::vector<double> >& Phi,
        const std::vector<std::vector<double> >& dPhi)
    {
        const int nr = static_cast<int>(radii.size()), nc = static_cast<int>(Phi.size());
        std::vector<double> flatPhi, flatDer;
        for(int c = 0; c < nc; c++) {
            flatPhi.insert(flatPhi.end(), Phi[c].begin(), Phi[c].end());
            flatDer.insert(flatDer.end(), dPhi[c].begin(), dPhi[c].end());
        }
        h = agama_createMultipoleFromCoefs(nr, radii.data(), nc, flatPhi.data(), flatDer.data());
        if(!h) throw std::runtime_error(agama_getError());
        readInfo();
    }
    virtual ~MultipoleB200() { agama_deletePotential(h); }

    virtual ::coord::SymmetryType symmetry() const { return sym; }
    virtual std::string name() const { return "Multipole"; }
    const agama_Potential* handle() const { return h; }

    /// potential, gradient and Hessian at n Cartesian points in one engine call (any output may
    /// be NULL), as n calls of eval(PosCar, ...)
    void evalmanyCar(size_t n, const ::coord::PosCar pos[], double pot[],
        ::coord::GradCar deriv[] = NULL, ::coord::HessCar deriv2[] = NULL, double time = 0) const
    {
        std::vector<double> x(3 * n), g(deriv ? 3 * n : 0), hh(deriv2 ? 6 * n : 0);
        for(size_t i = 0; i < n; i++) { x[3 * i] = pos[i].x; x[3 * i + 1] = pos[i].y; x[3 * i + 2] = pos[i].z; }
        detail::checkRef(agama_evalPotentialMany(h, static_cast<long>(n), x.data(), time, pot,
            deriv ? g.data() : NULL, deriv2 ? hh.data() : NULL));
        for(size_t i = 0; i < n; i++) {
            if(deriv) { deriv[i].dx = g[3 * i]; deriv[i].dy = g[3 * i + 1]; deriv[i].dz = g[3 * i + 2]; }
            if(deriv2) {
                const double* e = &hh[6 * i];
                deriv2[i].dx2 = e[0]; deriv2[i].dy2 = e[1]; deriv2[i].dz2 = e[2];
                deriv2[i].dxdy = e[3]; deriv2[i].dydz = e[4]; deriv2[i].dxdz = e[5];
            }
        }
    }

    /// the same at n cylindrical points, as n calls of eval(PosCyl, ...): evaluated in cylindrical
    /// coordinates on the engine, as the reference's Multipole::evalCyl does
    void evalmanyCyl(size_t n, const ::coord::PosCyl pos[], double pot[],
        ::coord::GradCyl deriv[] = NULL, ::coord::HessCyl deriv2[] = NULL, double time = 0) const
    {
        std::vector<double> x(3 * n), phi(n), g(deriv ? 3 * n : 0), hh(deriv2 ? 6 * n : 0);
        for(size_t i = 0; i < n; i++) { x[3 * i] = pos[i].R; x[3 * i + 1] = pos[i].z; x[3 * i + 2] = pos[i].phi; }
        detail::checkRef(agama_evalPotentialCylMany(h, static_cast<long>(n), x.data(), time, pot ? pot : phi.data(),
            deriv ? g.data() : NULL, deriv2 ? hh.data() : NULL));
        for(size_t i = 0; i < n; i++) {
            if(deriv) { deriv[i].dR = g[3 * i]; deriv[i].dz = g[3 * i + 1]; deriv[i].dphi = g[3 * i + 2]; }
            if(deriv2) {
                const double* q = &hh[6 * i];
                deriv2[i].dR2 = q[0]; deriv2[i].dz2 = q[1]; deriv2[i].dphi2 = q[2];
                deriv2[i].dRdz = q[3]; deriv2[i].dzdphi = q[4]; deriv2[i].dRdphi = q[5];
            }
        }
    }

    /// batched density (overrides the reference's per-point loop)
    virtual void evalmanyDensityCar(const size_t npoints, const ::coord::PosCar pos[],
        double values[], double time = 0) const
    {
        std::vector<double> x(3 * npoints);
        for(size_t i = 0; i < npoints; i++) { x[3 * i] = pos[i].x; x[3 * i + 1] = pos[i].y; x[3 * i + 2] = pos[i].z; }
        detail::checkRef(agama_evalDensityMany(h, static_cast<long>(npoints), x.data(), time, values));
    }
    virtual void evalmanyDensityCyl(const size_t npoints, const ::coord::PosCyl pos[],
        double values[], double time = 0) const
    {
        std::vector<double> x(3 * npoints);
        for(size_t i = 0; i < npoints; i++) {
            x[3 * i] = pos[i].R * std::cos(pos[i].phi); x[3 * i + 1] = pos[i].R * std::sin(pos[i].phi);
            x[3 * i + 2] = pos[i].z;
        }
        detail::checkRef(agama_evalDensityMany(h, static_cast<long>(npoints), x.data(), time, values));
    }

protected:
    virtual void evalCar(const ::coord::PosCar& pos, double* potential,
        ::coord::GradCar* deriv, ::coord::HessCar* deriv2, double time) const
    {
        double phi = 0;
        evalmanyCar(1, &pos, &phi, deriv, deriv2, time);
        if(potential) *potential = phi;
    }
    virtual void evalCyl(const ::coord::PosCyl& pos, double* potential,
        ::coord::GradCyl* deriv, ::coord::HessCyl* deriv2, double time) const
    {
        double phi = 0;
        evalmanyCyl(1, &pos, &phi, deriv, deriv2, time);
        if(potential) *potential = phi;
    }
    virtual double densityCar(const ::coord::PosCar& pos, double time) const
    {
        double rho = 0;
        evalmanyDensityCar(1, &pos, &rho, time);
        return rho;
    }
    virtual double densityCyl(const ::coord::PosCyl& pos, double time) const
    {
        double rho = 0;
        evalmanyDensityCyl(1, &pos, &rho, time);
        return rho;
    }

private:
    agama_Potential* h;
    ::coord::SymmetryType sym;
    void readInfo()
    {
        int lmax, mmax, symmetry, nr, nt;
        detail::checkRef(agama_getPotentialInfo(h, &lmax, &mmax, &symmetry, &nr, &nt));
        sym = static_cast<::coord::SymmetryType>(symmetry);
    }
    MultipoleB200(const MultipoleB200&);
    MultipoleB200& operator=(const MultipoleB200&);
};

/** The Staeckel-fudge action finder of a MultipoleB200 potential on the engine (focal-distance
    table built on the device), usable wherever the reference takes an actions::BaseActionFinder. */
class ActionFinderB200 : public actions::BaseActionFinder {
public:
    explicit ActionFinderB200(const std::shared_ptr<const MultipoleB200>& potential)
        : pot(potential), h(agama_createActionFinder(potential->handle()))
    {
        if(!h) throw std::runtime_error(agama_getError());
    }
    virtual ~ActionFinderB200() { agama_deleteActionFinder(h); }

    virtual std::string name() const { return "AxisymmetricFudge(potential=" + pot->name() + ")"; }

    virtual void eval(const ::coord::PosVelCyl& point, actions::Actions* act = NULL,
        actions::Angles* ang = NULL, actions::Frequencies* freq = NULL) const
    {
        evalmany(1, &point, act, ang, freq);
    }

    /// actions / angles / frequencies of n points in one engine call (any output may be NULL), as
    /// n calls of eval; unbound points give NaN as in the reference
    void evalmany(size_t n, const ::coord::PosVelCyl points[], actions::Actions act[] = NULL,
        actions::Angles ang[] = NULL, actions::Frequencies freq[] = NULL) const
    {
        if(!act && !ang && !freq) return;
        std::vector<double> x(6 * n), a(act ? 3 * n : 0), g(ang ? 3 * n : 0), f(freq ? 3 * n : 0);
        for(size_t i = 0; i < n; i++) {
            const double c = std::cos(points[i].phi), s = std::sin(points[i].phi);
            double* w = &x[6 * i];
            w[0] = points[i].R * c; w[1] = points[i].R * s; w[2] = points[i].z;
            w[3] = points[i].vR * c - points[i].vphi * s; w[4] = points[i].vR * s + points[i].vphi * c;
            w[5] = points[i].vz;
        }
        if(ang || freq)
            detail::checkRef(agama_evalActionsAnglesFrequenciesMany(h, static_cast<long>(n), x.data(),
                act ? a.data() : NULL, ang ? g.data() : NULL, freq ? f.data() : NULL));
        else
            detail::checkRef(agama_evalActionsMany(h, static_cast<long>(n), x.data(), a.data(), NULL));
        for(size_t i = 0; i < n; i++) {
            if(act) act[i] = actions::Actions(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
            if(ang) ang[i] = actions::Angles(g[3 * i], g[3 * i + 1], g[3 * i + 2]);
            if(freq) freq[i] = actions::Frequencies(f[3 * i], f[3 * i + 1], f[3 * i + 2]);
        }
    }

private:
    std::shared_ptr<const MultipoleB200> pot;
    agama_ActionFinder* h;
};

}  // namespace agama_b200

#endif
