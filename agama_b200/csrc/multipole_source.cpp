// A Multipole potential from a density model: the Poisson solve in spherical harmonics.
//
// Reference: createMultipole (src/potential_multipole.cpp:1400-1441) -> chooseGridRadii (:369-484),
// createExpGrid (src/math_spline.cpp:4223-4234), computePotentialCoefsFromSource (:1013-1114) over
// computeSphHarmCoefs (:239-285, SphHarmTransformForward, src/math_sphharm.cpp:266-384) and
// restrictSphHarmCoefs (:151-185), with the density models the factory builds for
// "density=<type>" (src/potential_factory.cpp:476-516, :1337-1353): Dehnen, Plummer, NFW,
// MiyamotoNagai, Spheroid and Disk, and their sum.  Host code, run once per potential; the
// result is the set of coefficients Phi_lm(r_k), dPhi_lm/dr(r_k) that the Multipole tables are
// built from.
#include "multipole.h"
#include "sphharm.cuh"
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>

namespace agb {

namespace {

/// the cube root of the double-precision epsilon to the digits the reference uses (ROOT3_DBL_EPSILON)
constexpr double ROOT3_EPS = 6.0554544523933429e-06;

double pow2d(double x) { return x * x; }
double pow3d(double x) { return x * x * x; }

/// x^n with the shortcuts of the reference's math::pow(double, double) (src/math_core.cpp:135-147)
double powr(double x, double n)
{
    if(n == 0.0) return 1;
    if(n == 1.0) return x;
    if(n == -1.0) return 1 / x;
    if(n == 2.0) return x * x;
    if(n == -2.0) return 1 / (x * x);
    if(n == 0.5) return sqrt(x);
    if(n == -0.5) return 1 / sqrt(x);
    if(n == 3.0) return x * x * x;
    if(n == -3.0) return 1 / (x * x * x);
    return std::pow(x, n);
}

// ---------------------------------------------------------------------------------------------
// density models (value at a cylindrical point), with the symmetry flags of the reference's classes

struct DensityModel {
    virtual ~DensityModel() {}
    virtual int symmetry() const = 0;
    virtual double density(double R, double z, double phi) const = 0;
};

/// Dehnen: rho = M a (3 - gamma) / (4 pi p q) m^-gamma (a + m)^(gamma - 4), m^2 = x^2 + (y/p)^2 + (z/q)^2
/// (Dehnen::densityCar, src/potential_dehnen.cpp:37-42)
struct DehnenModel : DensityModel {
    double mass, a, gamma, p, q;
    int symmetry() const override { return p == 1 && q == 1 ? SYM_SPHERICAL : p == 1 ? SYM_AXISYMMETRIC : SYM_TRIAXIAL; }
    double density(double R, double z, double phi) const override
    {
        const double x = R * cos(phi), y = R * sin(phi);
        const double m = sqrt(pow2d(x) + pow2d(y / p) + pow2d(z / q));
        return mass * a * (3 - gamma) / (4 * M_PI * p * q) * powr(m, -gamma) * powr(a + m, gamma - 4);
    }
};

/// Plummer (Plummer::densitySph, src/potential_analytic.cpp:21-25)
struct PlummerModel : DensityModel {
    double mass, b;
    int symmetry() const override { return SYM_SPHERICAL; }
    double density(double R, double z, double) const override
    {
        const double r = sqrt(R * R + z * z), invrsq = 1. / (pow2d(r) + pow2d(b));
        return 3. / 4 / M_PI * mass * pow2d(b * invrsq) * sqrt(invrsq);
    }
};

/// NFW (NFW::densitySph, src/potential_analytic.h:67-68)
struct NFWModel : DensityModel {
    double mass, rs;
    int symmetry() const override { return SYM_SPHERICAL; }
    double density(double R, double z, double) const override
    {
        const double r = sqrt(R * R + z * z);
        return (1. / 4 / M_PI) * mass / r / pow2d(r + rs);
    }
};

/// Miyamoto-Nagai (MiyamotoNagai::densityCyl, src/potential_analytic.cpp:104-110)
struct MiyamotoNagaiModel : DensityModel {
    double mass, a, b;
    int symmetry() const override { return SYM_AXISYMMETRIC; }
    double density(double R, double z, double) const override
    {
        const double zb = sqrt(pow2d(z) + pow2d(b));
        const double azb2 = pow2d(a + zb), R2azb2 = pow2d(R) + azb2;
        return 1. / 4 / M_PI * mass * pow2d(b) * (a + 3 * zb * azb2 / R2azb2) / (pow3d(zb) * R2azb2 * sqrt(R2azb2));
    }
};

/// Spheroid: rho0 (r/a)^-gamma (1 + (r/a)^alpha)^((gamma-beta)/alpha) exp(-(r/rcut)^xi) at the
/// ellipsoidal radius (SpheroidDensityFnc and SpheroidDensity::densityCyl,
/// src/potential_spheroid.cpp:34-47, :261-266); rho0 from the total mass (SpheroidParam::mass:
/// the Beta-function expression without a cutoff, src/potential_spheroid.cpp:117-129)
struct SpheroidModel : DensityModel {
    double rho0 = 0, a = 1, rcut = INFINITY, xi = 2, alpha = 1, beta = 4, gamma = 1, p = 1, q = 1;
    int symmetry() const override { return p == 1 && q == 1 ? SYM_SPHERICAL : p == 1 ? SYM_AXISYMMETRIC : SYM_TRIAXIAL; }
    double profile(double r) const
    {
        const double r0 = r / a;
        double rho = rho0 * powr(r0, -gamma) * powr(1 + powr(r0, alpha), (gamma - beta) / alpha);
        if(rcut < INFINITY) rho *= exp(-powr(r / rcut, xi));
        return rho;
    }
    double density(double R, double z, double phi) const override
    {
        const double p2 = p * p, q2 = q * q;
        const double R2 = p2 == 1 ? pow2d(R) : pow2d(R) * (1 + pow2d(sin(phi)) * (1 / p2 - 1));
        return profile(sqrt(R2 + pow2d(z) / q2));
    }
    /// total mass for rho0 = 1 (only the case without a cutoff has a closed form)
    double unitMass() const
    {
        if(rcut < INFINITY)
            throw std::invalid_argument("Spheroid with an outer cutoff: give densityNorm instead of mass");
        if(beta <= 3) throw std::invalid_argument("Spheroid model has infinite mass (provide densityNorm instead)");
        if(gamma >= 3 || alpha <= 0) throw std::invalid_argument("Spheroid: invalid parameters");
        return 4 * M_PI * pow3d(a) * p * q *
            (std::tgamma((beta - 3) / alpha) * std::tgamma((3 - gamma) / alpha) / std::tgamma((beta - gamma) / alpha) / alpha);
    }
};

/// Disk: Sigma0 exp(-R/Rd) times the vertical profile h(z): exponential (hz > 0),
/// isothermal sech^2 (hz < 0) or thin (hz = 0) (DiskDensity::densityCyl with
/// DiskDensityRadialExp and DiskDensityVertical*, src/potential_disk.cpp:36-53, :113-165, :205-210);
/// Sigma0 from the total mass M = 2 pi Rd^2 Sigma0 (DiskParam::mass, :190-203)
struct DiskModel : DensityModel {
    double sigma0 = 0, Rd = 1, hz = 0.1;
    int symmetry() const override { return SYM_AXISYMMETRIC; }
    double density(double R, double z, double) const override
    {
        double h;
        if(hz > 0) {
            const double inv = 1. / hz, x = fabs(z * inv);
            h = 0.5 * exp(-x) * inv;
        } else if(hz < 0) {
            const double inv = 1. / -hz, x = fabs(z * inv), e = exp(-x), inv1 = 1. / (1 + e);
            h = e * inv * pow2d(inv1);
        } else
            h = 0;
        return sigma0 * exp(-R * (1. / Rd)) * h;
    }
};

/// a sum of density models (CompositeDensity: components summed in order; the symmetry common
/// to all of them)
struct CompositeModel : DensityModel {
    std::vector<std::unique_ptr<DensityModel>> comps;
    int symmetry() const override
    {
        int s = SYM_SPHERICAL;
        for(auto& c : comps) s &= c->symmetry();
        return s;
    }
    double density(double R, double z, double phi) const override
    {
        double sum = 0;
        for(auto& c : comps) sum += c->density(R, z, phi);
        return sum;
    }
};

std::string lowerStr(std::string s) { for(auto& c : s) c = static_cast<char>(tolower(c)); return s; }

double getNum(const std::map<std::string, std::string>& kv, const std::string& key, double def)
{
    auto it = kv.find(key);
    if(it == kv.end()) return def;
    char* end = nullptr;
    const double v = strtod(it->second.c_str(), &end);
    if(end == it->second.c_str()) throw std::invalid_argument("parameter " + key + ": not a number");
    return v;
}

/// one density model from its key=value parameters (names as in the reference's factory, case-insensitive)
std::unique_ptr<DensityModel> makeModel(const std::map<std::string, std::string>& kv)
{
    auto t = kv.find("type");
    if(t == kv.end()) throw std::invalid_argument("density: no type given");
    const std::string type = lowerStr(t->second);
    const double mass = getNum(kv, "mass", 1), a = getNum(kv, "scaleradius", 1);
    if(type == "dehnen") {
        auto m = std::make_unique<DehnenModel>();
        m->mass = mass; m->a = a; m->gamma = getNum(kv, "gamma", 1);
        m->p = getNum(kv, "axisratioy", 1); m->q = getNum(kv, "axisratioz", 1);
        if(m->gamma < 0 || m->gamma > 2 || !(m->p > 0) || !(m->q > 0))
            throw std::invalid_argument("Dehnen: invalid parameters");
        return m;
    }
    if(type == "plummer") {
        auto m = std::make_unique<PlummerModel>();
        m->mass = mass; m->b = a;
        return m;
    }
    if(type == "nfw") {
        auto m = std::make_unique<NFWModel>();
        m->mass = mass; m->rs = a;
        return m;
    }
    if(type == "miyamotonagai") {
        auto m = std::make_unique<MiyamotoNagaiModel>();
        m->mass = mass; m->a = a; m->b = getNum(kv, "scaleheight", 0);
        return m;
    }
    if(type == "spheroid") {
        auto m = std::make_unique<SpheroidModel>();
        m->a = a; m->alpha = getNum(kv, "alpha", 1); m->beta = getNum(kv, "beta", 4); m->gamma = getNum(kv, "gamma", 1);
        m->rcut = getNum(kv, "outercutoffradius", INFINITY); m->xi = getNum(kv, "cutoffstrength", 2);
        m->p = getNum(kv, "axisratioy", 1); m->q = getNum(kv, "axisratioz", 1);
        const double norm = getNum(kv, "densitynorm", NAN);
        m->rho0 = std::isfinite(norm) ? norm : mass / m->unitMass();
        return m;
    }
    if(type == "disk") {
        auto m = std::make_unique<DiskModel>();
        m->Rd = a; m->hz = getNum(kv, "scaleheight", 0.1);
        if(kv.count("innercutoffradius") || kv.count("modulationamplitude") || kv.count("sersicindex"))
            throw std::invalid_argument("Disk: only the exponential profile (no inner cutoff, modulation or Sersic index)");
        if(!(m->Rd > 0)) throw std::invalid_argument("Disk scale radius cannot be <=0");
        const double sd = getNum(kv, "surfacedensity", NAN);
        // DiskParam::mass with unit surface density: pi Rd^2 Gamma(2 n + 1), n = 1
        m->sigma0 = std::isfinite(sd) ? sd : mass / (M_PI * pow2d(m->Rd) * std::tgamma(3.0));
        return m;
    }
    throw std::invalid_argument("density type '" + t->second + "' is not supported by the engine's Multipole "
        "construction (Dehnen, Plummer, NFW, MiyamotoNagai, Spheroid, Disk)");
}

// ---------------------------------------------------------------------------------------------
// spherical average of a density (Sphericalized<BaseDensity>::value, src/potential_base.cpp:424-431,
// over sphericalAverage, :205-260: 8 Gauss-Radau nodes in cos(theta) on [0, 1] (the last at 0),
// 8 or 17 azimuths, the z < 0 half and the y < 0 half folded in by symmetry)

// the Gauss-Radau rule of the reference's sphericalAverage (same 16-digit nodes and weights, so
// that the grid radii chosen from it are the same)
const double RADAU_COS[8] = { 0.9775206135612875, 0.8853209468390958, 0.7342101772154106,
    0.5471536263305554, 0.3526247171131696, 0.1802406917368924, 0.0562625605369222, 0 };
const double RADAU_SIN[8] = { 0.2108398682952634, 0.4649804523718464, 0.6789222456756852,
    0.8370322031996875, 0.9357648256270681, 0.9836225358551961, 0.9984160076249926, 1 };
const double RADAU_W[8] = { 0.02862720368606458, 0.06241197533246655, 0.08675369890862478,
    0.09789304186312342, 0.09412938634727970, 0.07603265516169632, 0.04633953870074772, 0.015625 };

double sphericalDensity(const DensityModel& d, double r)
{
    const int sym = d.symmetry();
    if((sym & SYM_SPHERICAL) == SYM_SPHERICAL || r == 0 || r == INFINITY) return d.density(r, 0, 0);
    const int nphi = 8;
    const bool ysym = (sym & SYM_YREFL) == SYM_YREFL, zsym = (sym & SYM_ZREFL) == SYM_ZREFL;
    const int Nphi = (sym & SYM_ZROT) == SYM_ZROT ? 1 : ysym ? nphi + 1 : 2 * nphi + 1;
    const int Ntheta = zsym ? 8 : 15;
    double result = 0;
    for(int ith = 0; ith < Ntheta; ith++) {
        const double cth = RADAU_COS[ith % 8] * (ith < 8 ? 1 : -1), sth = RADAU_SIN[ith % 8];
        for(int iph = 0; iph < Nphi; iph++) {
            const double w = RADAU_W[ith % 8] * (zsym && ith < 7 ? 2 : 1) * (ysym && iph > 0 ? 2 : 1);
            result += d.density(r * sth, r * cth, M_PI / (nphi + 0.5) * iph) * w;
        }
    }
    if(Nphi > 1) result *= 1. / (2 * nphi + 1);
    return result;
}

/** the radial grid of a density model when rmin or rmax is not given (chooseGridRadii,
    src/potential_multipole.cpp:369-484): a sweep in ln r from 0 in steps +-LOGSTEP finds the
    radius of largest density-weighted logarithmic curvature; rmax and rmin are set around it, and
    rmin is moved out while Phi(r) - Phi(0) is below 4e-11 of Phi(0) */
void chooseGridRadii(const DensityModel& src, int gridSizeR, double& rmin, double& rmax)
{
    if(rmax != 0 && rmin != 0) return;
    const double LOGSTEP = log(1 + sqrt(20. / gridSizeR)), LOGRMAX = 100.,
        DELTA = ROOT3_EPS * 0.99, MAXRHO = 1e100, MINRHO = 1e-100;
    double logr = 0., maxcurv = 0., rcenter = 1.;
    int skipped = 0;
    std::vector<double> rad, rho;
    while(fabs(logr) < LOGRMAX) {
        const double r = exp(logr), rho0 = sphericalDensity(src, r);
        double curv = 0;
        if(fabs(rho0) >= MINRHO && fabs(rho0) <= MAXRHO) {
            if(logr > 0) { rad.push_back(r); rho.push_back(rho0); }
            else { rad.insert(rad.begin(), r); rho.insert(rho.begin(), rho0); }
            const double rhop = sphericalDensity(src, exp(logr + DELTA));
            const double rhom = sphericalDensity(src, exp(logr - DELTA));
            const double derp = log(rhop / rho0) / DELTA, derm = log(rho0 / rhom) / DELTA;
            double der2 = fabs(derp - derm) / DELTA;
            if(der2 < 10 * DELTA) der2 = 0;
            curv = der2 * rho0 * pow2d(r);
        }
        if(curv > maxcurv) { skipped = 0; maxcurv = curv; rcenter = r; }
        else if(++skipped > gridSizeR) break;
        logr = -logr + (logr > 0 ? 0. : LOGSTEP);
    }
    if(rad.size() < 2) {
        rad.insert(rad.begin(), exp(-LOGSTEP)); rho.insert(rho.begin(), 0.0);
        rad.push_back(exp(LOGSTEP)); rho.push_back(0.0);
    }
    if(rmax == 0) rmax = fmin(rad.back(), rcenter * exp(LOGSTEP * 0.5 * gridSizeR));
    if(rmin == 0) {
        rmin = fmax(rad[0], rmax * exp(-LOGSTEP * gridSizeR));
        const double DELTAPHI = pow2d(ROOT3_EPS);
        double Phi0 = 0;
        for(size_t i = 1; i < rad.size(); i++)
            Phi0 += -4 * M_PI / 6 * (rad[i] - rad[i - 1]) *
                (rho[i] * (2 * rad[i] + rad[i - 1]) + rho[i - 1] * (rad[i] + 2 * rad[i - 1]));
        double enclMass = 0, deltaPhi = 0;
        for(size_t i = 1; i < rad.size() && rad[i] < rmax * 0.999; i++) {
            enclMass += 4 * M_PI / 12 * (rad[i] - rad[i - 1]) *
                ((rho[i] + rho[i - 1]) * pow2d(rad[i] + rad[i - 1]) + 2 * rho[i] * pow2d(rad[i]) +
                 2 * rho[i - 1] * pow2d(rad[i - 1]));
            deltaPhi += 4 * M_PI / 6 * (rad[i] - rad[i - 1]) *
                (rho[i] * (2 * rad[i] + rad[i - 1]) + rho[i - 1] * (rad[i] + 2 * rad[i - 1]));
            const double dPhi = enclMass / rad[i] + deltaPhi;
            if(fabs(dPhi) < fabs(Phi0) * DELTAPHI) rmin = rad[i];
        }
    }
}

/** forward spherical-harmonic transform of values on the angular grid of indices ind
    (SphHarmTransformForward, src/math_sphharm.cpp:266-384): Gauss-Legendre nodes of order lmax+1
    in cos(theta) (only the z >= 0 half under z-reflection symmetry), mmax+1 azimuths
    phi_k = pi k / (mmax + 1/2) (2 mmax + 1 when sines are needed) */
struct ForwardTransform {
    HarmIndices ind;
    int ngrid, ntheta, nphi, nfour;
    bool useSine, zsym;
    std::vector<double> cosTheta, legFnc, trigFnc;
    explicit ForwardTransform(const HarmIndices& I) : ind(I)
    {
        ngrid = ind.lmax + 1;
        ntheta = ind.lmax / 2 + 1;
        useSine = ind.mmin() < 0;
        nfour = useSine ? 2 * ind.mmax + 1 : ind.mmax + 1;
        nphi = nfour;
        zsym = (ind.sym & SYM_ZREFL) == SYM_ZREFL;
        std::vector<double> nodes(ngrid), weights(ngrid);
        glNodesWeights(ngrid, nodes.data(), weights.data());
        cosTheta.resize(ngrid);
        const int nlegfn = (ind.lmax + 1) * (ind.mmax + 1);
        legFnc.assign(static_cast<size_t>(ntheta) * nlegfn, 0);
        for(int j = 0; j < ngrid; j++) {
            cosTheta[j] = nodes[ngrid - 1 - j];
            if(j >= ntheta) continue;
            for(int m = 0; m <= ind.mmax; m++) {
                const double tau = cosTheta[j] / (sqrt(1 - pow2d(cosTheta[j])) + 1);
                double* P = &legFnc[static_cast<size_t>(j) * nlegfn + m * (ind.lmax + 1) + m];
                legendreArray(ind.lmax, m, tau, P, nullptr, nullptr);
                for(int l = m; l <= ind.lmax; l++)
                    P[l - m] *= weights[ngrid - 1 - j] * (0.5 / SQRT_PI) * (m > 0 ? M_SQRT2 : 1);
            }
        }
        // azimuthal weights: uniform grid, cos (and sin) of m phi_k
        const int nfnc = nfour, nph = ind.mmax + 1;
        trigFnc.assign(static_cast<size_t>(nph) * nfnc, 0);
        const double weight = M_PI / (ind.mmax + 0.5);
        for(int k = 0; k < nph; k++) {
            trigFnc[k * nfnc] = 1.;
            if(ind.mmax > 0) trigMultiAngle(phiNode(k), ind.mmax, useSine, &trigFnc[k * nfnc + 1]);
            for(int m = 0; m < nfnc; m++) trigFnc[k * nfnc + m] *= weight * (useSine || k == 0 ? 1 : 2);
        }
    }
    double phiNode(int k) const { return k * M_PI / (ind.mmax + 0.5); }
    int thetaSize() const { return zsym ? ntheta : ngrid; }
    int size() const { return thetaSize() * nphi; }
    /// the angular points: theta index j (cos theta = cosTheta[j]), azimuth index k
    double pointCos(int a) const { return cosTheta[a / nphi]; }
    double pointPhi(int a) const { return phiNode(a % nphi); }
    void transform(const double* values, double* coefs) const
    {
        if(ind.size() == 1) { coefs[0] = values[0]; return; }
        std::fill(coefs, coefs + ind.size(), 0.);
        const int mmin = ind.mmin(), nsamp = thetaSize();
        std::vector<double> valm(static_cast<size_t>(nsamp) * nfour);
        for(int j = 0; j < nsamp; j++) {
            const double* v = values + static_cast<size_t>(j) * nphi;
            double* out = &valm[static_cast<size_t>(j) * nfour];
            for(int mm = 0; mm < nfour; mm++) {
                out[mm] = 0;
                const int m = useSine ? mm - ind.mmax : mm;
                for(int k = 0; k < nfour; k++) {
                    const int indphi = k <= ind.mmax ? k : 2 * ind.mmax + 1 - k;
                    const int indfnc = m >= 0 ? m : ind.mmax - m;
                    double fnc = trigFnc[indphi * nfour + indfnc];
                    if(m < 0 && k > ind.mmax) fnc *= -1;
                    out[mm] += fnc * v[k];
                }
            }
        }
        const int nlegfn = (ind.lmax + 1) * (ind.mmax + 1);
        for(int m = ind.mmin(); m <= ind.mmax; m++) {
            for(int l = ind.lmin(m); l <= ind.lmax; l += ind.step) {
                const int c = HarmIndices::index(l, m), absm = abs(m);
                for(int j = 0; j < ngrid; j++) {
                    const int jsamp = j < nsamp ? j : ngrid - 1 - j;
                    const int absj = j < ntheta ? j : ind.lmax - j;
                    double Plm = legFnc[static_cast<size_t>(absj) * nlegfn + absm * (ind.lmax + 1) + l];
                    if((l + m) % 2 == 1 && j > ind.lmax / 2) Plm *= -1;
                    coefs[c] += Plm * valm[static_cast<size_t>(jsamp) * nfour + m - mmin];
                }
            }
        }
    }
};

/// spherical-harmonic coefficients of the density at the given radii (computeSphHarmCoefs for a
/// density source, src/potential_multipole.cpp:239-285): coefs[c][k], near-zero terms (below 1e-10
/// of the largest at each radius) set to zero
std::vector<std::vector<double>> densityCoefs(const DensityModel& src, const HarmIndices& ind,
    const std::vector<double>& radii)
{
    const ForwardTransform tr(ind);
    const int na = tr.size();
    std::vector<std::vector<double>> coefs(ind.size(), std::vector<double>(radii.size(), 0));
    std::vector<double> values(na), sh(ind.size());
    for(size_t k = 0; k < radii.size(); k++) {
        for(int a = 0; a < na; a++) {
            const double ct = tr.pointCos(a), r = radii[k];
            values[a] = src.density(r * sqrt(1 - pow2d(ct)), r * ct, tr.pointPhi(a));
        }
        tr.transform(values.data(), sh.data());
        double mag = 0;
        for(double v : sh) mag = fmax(mag, fabs(v));
        mag *= 1e-10;
        for(double& v : sh) if(fabs(v) <= mag) v = 0;
        for(int c = 0; c < ind.size(); c++) coefs[c][k] = sh[c];
    }
    return coefs;
}

/** Phi_lm(r_k) and dPhi_lm/dr(r_k) from the density coefficients by Gauss-Legendre quadrature of
    order 10 on every radial segment (the last one to infinity in t = r_{N-1} / r), with the
    interior and exterior integrals accumulated through the recurrences in (r_k / r_{k-1})^n
    (computePotentialCoefsFromSource, src/potential_multipole.cpp:1013-1114) */
void potentialCoefs(const DensityModel& src, const HarmIndices& ind, const std::vector<double>& gridRadii,
    std::vector<std::vector<double>>& Phi, std::vector<std::vector<double>>& dPhi)
{
    const int N = static_cast<int>(gridRadii.size()), GLORDER = 10;
    double glnodes[GLORDER], glweights[GLORDER];
    glNodesWeights(GLORDER, glnodes, glweights);
    for(int s = 0; s < GLORDER; s++) { glnodes[s] = 0.5 * (glnodes[s] + 1); glweights[s] *= 0.5; }  // on [0, 1]
    std::vector<double> intRadii((N + 1) * GLORDER);
    for(int k = 0; k <= N; k++) {
        const double rkm1 = k > 0 ? gridRadii[k - 1] : 0, delta = k < N ? gridRadii[k] - rkm1 : gridRadii.back();
        for(int s = 0; s < GLORDER; s++)
            intRadii[k * GLORDER + s] = k < N ? rkm1 + glnodes[s] * delta : gridRadii.back() / glnodes[s];
    }
    const std::vector<std::vector<double>> ic = densityCoefs(src, ind, intRadii);
    Phi.assign(ind.size(), std::vector<double>(N, 0.));
    dPhi.assign(ind.size(), std::vector<double>(N, 0.));
    std::vector<double> Pint(N), Pext(N);
    for(int m = ind.mmin(); m <= ind.mmax; m++) {
        for(int l = ind.lmin(m); l <= ind.lmax; l += ind.step) {
            const int c = HarmIndices::index(l, m);
            for(int k = 0; k < N; k++) {
                double integr = 0;
                for(int s = 0; s < GLORDER; s++)
                    integr += ic[c][k * GLORDER + s] * glweights[s] * powr(intRadii[k * GLORDER + s] / gridRadii[k], l + 2);
                Pint[k] = integr * (gridRadii[k] - (k > 0 ? gridRadii[k - 1] : 0)) * gridRadii[k] +
                    (k > 0 ? Pint[k - 1] * powr(gridRadii[k - 1] / gridRadii[k], l + 1) : 0);
            }
            {
                double integr = 0;
                for(int s = 0; s < GLORDER; s++)
                    integr += ic[c][N * GLORDER + s] * glweights[s] *
                        powr(intRadii[N * GLORDER + s] / gridRadii[N - 1], 1 - l) / pow2d(glnodes[s]);
                Pext[N - 1] = integr * gridRadii[N - 1] * gridRadii[N - 1];
            }
            for(int k = N - 2; k >= 0; k--) {
                double integr = 0;
                for(int s = 0; s < GLORDER; s++)
                    integr += ic[c][(k + 1) * GLORDER + s] * glweights[s] *
                        powr(intRadii[(k + 1) * GLORDER + s] / gridRadii[k], 1 - l);
                Pext[k] = integr * (gridRadii[k + 1] - gridRadii[k]) * gridRadii[k] +
                    Pext[k + 1] * powr(gridRadii[k] / gridRadii[k + 1], l);
            }
            const double mul = -4 * M_PI / (2 * l + 1);
            for(int k = 0; k < N; k++) {
                Phi[c][k] = mul * (Pint[k] + Pext[k]);
                dPhi[c][k] = mul * (-(l + 1) * Pint[k] + l * Pext[k]) / gridRadii[k];
            }
        }
    }
}

/// indices of the source expansion: as makeIndices, but lmax may exceed the evaluators' limit
/// (the source is expanded to lmax + 6 for the angular quadrature); mmax stays within it
HarmIndices sourceIndices(int lmax, int mmax, int sym)
{
    if(lmax > 2 * LMAX_MAX || mmax > LMAX_MAX || mmax > lmax)
        throw std::invalid_argument("Multipole: order of the source expansion too large");
    HarmIndices h;
    h.lmax = lmax; h.mmax = mmax;
    h.step = ((sym & SYM_ZREFL) == SYM_ZREFL || (sym & SYM_REFL) == SYM_REFL) ? 2 : 1;
    if(mmax == 0) sym |= SYM_ZROT | SYM_XREFL | SYM_YREFL;
    if(lmax == 0) sym |= SYM_ROT | SYM_ZREFL | SYM_REFL;
    h.sym = sym;
    const bool xrefl = (sym & SYM_XREFL) == SYM_XREFL, yrefl = (sym & SYM_YREFL) == SYM_YREFL,
        refl = (sym & SYM_REFL) == SYM_REFL, bisym = (sym & (SYM_XREFL | SYM_YREFL | SYM_REFL)) == (SYM_XREFL | SYM_YREFL | SYM_REFL);
    for(int m = -mmax; m <= mmax; m++) {
        int lm = abs(m);
        if(refl && m % 2 != 0) lm = abs(m) + 1;
        if((yrefl && m < 0) || (xrefl && ((m < 0) ^ (m % 2 != 0))) || (bisym && m % 2 != 0)) lm = lmax + 1;
        h.lminArr[m + mmax] = lm;
    }
    return h;
}

int symmetryFromName(const std::string& s)
{
    const std::string v = lowerStr(s);
    if(v.empty()) return -1;
    if(v[0] == 's') return SYM_SPHERICAL;
    if(v[0] == 'a') return SYM_AXISYMMETRIC;
    if(v[0] == 't') return SYM_TRIAXIAL;
    if(v[0] == 'n') return SYM_NONE;
    if(v[0] == 'b') return SYM_XREFL | SYM_YREFL | SYM_REFL;
    if(v[0] == 'r') return SYM_REFL;
    char* end = nullptr;
    const long n = strtol(v.c_str(), &end, 10);
    if(end == v.c_str()) throw std::invalid_argument("unknown symmetry '" + s + "'");
    return static_cast<int>(n);
}

}  // namespace

void multipoleCoefsFromDensity(const std::vector<std::map<std::string, std::string>>& densities,
    const std::map<std::string, std::string>& params, std::vector<double>& radii,
    std::vector<std::vector<double>>& Phi, std::vector<std::vector<double>>& dPhi)
{
    if(densities.empty()) throw std::invalid_argument("Multipole: no density given");
    CompositeModel composite;
    for(const auto& kv : densities) composite.comps.push_back(makeModel(kv));
    const DensityModel& src = composite.comps.size() == 1 ? *composite.comps[0] : composite;
    int lmax = static_cast<int>(getNum(params, "lmax", 6));
    int mmax = static_cast<int>(getNum(params, "mmax", lmax));
    const int gridSizeR = static_cast<int>(getNum(params, "gridsizer", 25));
    double rmin = getNum(params, "rmin", 0), rmax = getNum(params, "rmax", 0);
    const bool fixOrder = getNum(params, "fixorder", 0) != 0;
    auto symIt = params.find("symmetry");
    int symExp = symIt == params.end() ? -1 : symmetryFromName(symIt->second);
    // createMultipole (src/potential_multipole.cpp:1400-1441)
    if(gridSizeR < 2 || !(rmin >= 0) || !(rmax == 0 || rmax > rmin))
        throw std::invalid_argument("Multipole: invalid grid parameters");
    if(lmax < 0 || mmax < 0 || mmax > lmax || lmax > LMAX_MAX)
        throw std::invalid_argument("Multipole: invalid choice of expansion order");
    const int symSrc = src.symmetry();
    symExp = symExp < 0 ? symSrc : (symSrc | symExp);
    chooseGridRadii(src, gridSizeR, rmin, rmax);
    // createExpGrid (src/math_spline.cpp:4223-4234)
    radii.assign(gridSizeR, 0);
    {
        const double logmin = log(rmin), logmax = log(rmax);
        radii.front() = rmin;
        radii.back() = rmax;
        for(int k = 1; k < gridSizeR - 1; k++) radii[k] = exp(logmin + k * (logmax - logmin) / (gridSizeR - 1));
    }
    int lmaxSrc = fixOrder ? lmax : std::max(lmax + 6, 12);
    int mmaxSrc = fixOrder ? mmax : std::max(mmax + 6, 12);
    if((symSrc & SYM_SPHERICAL) == SYM_SPHERICAL) lmaxSrc = 0;
    if((symSrc & SYM_ZROT) == SYM_ZROT) mmaxSrc = 0;
    if((symExp & SYM_SPHERICAL) == SYM_SPHERICAL) lmax = 0;
    if((symExp & SYM_ZROT) == SYM_ZROT) mmax = 0;
    // the engine's index tables hold azimuthal orders up to LMAX_MAX: the source's angular
    // quadrature is capped there (the reference goes to mmax + 6 for mmax > LMAX_MAX - 6)
    lmaxSrc = std::min(lmaxSrc, 2 * LMAX_MAX);
    mmaxSrc = std::min(std::min(mmaxSrc, lmaxSrc), LMAX_MAX);
    const HarmIndices indSrc = sourceIndices(lmaxSrc, mmaxSrc, symSrc);
    potentialCoefs(src, indSrc, radii, Phi, dPhi);
    // restrictSphHarmCoefs (src/potential_multipole.cpp:151-185)
    const HarmIndices indOut = makeIndices(lmax, mmax, symExp);
    std::vector<bool> keep(indOut.size(), false);
    for(int m = indOut.mmin(); m <= mmax; m++)
        for(int l = indOut.lmin(m); l <= lmax; l += indOut.step) keep[HarmIndices::index(l, m)] = true;
    int lmaxActual = 0;
    for(size_t c = 0; c < Phi.size(); c++) {
        const int l = static_cast<int>(floor(sqrt(static_cast<double>(c)))), m = static_cast<int>(c) - l * (l + 1);
        bool isZero = true;
        if(l > lmax || abs(m) > mmax || !keep[c]) {
            std::fill(Phi[c].begin(), Phi[c].end(), 0.);
            std::fill(dPhi[c].begin(), dPhi[c].end(), 0.);
        } else {
            for(double v : Phi[c]) isZero &= v == 0;
            for(double v : dPhi[c]) isZero &= v == 0;
        }
        if(!isZero) lmaxActual = std::max(lmaxActual, l);
    }
    const size_t n = static_cast<size_t>(lmaxActual + 1) * (lmaxActual + 1);
    if(Phi.size() > n) { Phi.resize(n); dPhi.resize(n); }
}

}  // namespace agb
