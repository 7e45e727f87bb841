"""Seeded synthetic inputs of the benchmark configurations (numpy PCG64 generators).

The samplers need the potential only through small callables (potential / force at points),
so the same code produces the inputs for the engine (with its own Potential) and for the
test fixtures (with the reference oracle).

  config 1: triaxial Dehnen gamma=1 (a=1, axis ratios 1:0.8:0.6) Multipole lmax=6, 50 nodes,
            r in [1e-3, 1e3]; 1e5 force points from the density; 1e4 orbits with
            |v| = u v_esc(r), u ~ U[0.2, 0.8], isotropic directions, T = 10 T_circ(E).
  config 2: Miyamoto-Nagai disk (M=0.1, a=3, b=0.3) + NFW halo (M=1, rs=20), axisymmetric
            Multipole lmax=8, 60 nodes; 1e6 disk-like particles.
  config 3: triaxial Dehnen gamma=0.5 (1:0.7:0.5) Multipole lmax=8, 64 nodes, Omega=0.05;
            1e5 orbits with T log-uniform over 10-1000 T_circ.
  config 4: the config-1 potential axisymmetrised (lmax=6, mmax=0); MLP-bracketed fudge.
  config 5: Spheroid (q=0.6, gamma=1, beta=4, M=1) + exponential disk (M=0.05, Rd=3, hz=0.3),
            axisymmetric Multipole lmax=12, 80 nodes; 1e6 orbits x 100 T_circ, then actions.
"""
import numpy as np

# parameters of the Multipole potentials, in the reference's key=value vocabulary
CONFIG_POTENTIALS = {
    1: dict(density=dict(type="Dehnen", mass=1, scaleRadius=1, gamma=1, axisRatioY=0.8, axisRatioZ=0.6),
            lmax=6, gridSizeR=50, rmin=1e-3, rmax=1e3, symmetry="triaxial"),
    2: dict(density=[dict(type="MiyamotoNagai", mass=0.1, scaleRadius=3, scaleHeight=0.3),
                     dict(type="NFW", mass=1, scaleRadius=20)],
            lmax=8, gridSizeR=60, symmetry="axisymmetric"),
    3: dict(density=dict(type="Dehnen", mass=1, scaleRadius=1, gamma=0.5, axisRatioY=0.7, axisRatioZ=0.5),
            lmax=8, gridSizeR=64, symmetry="triaxial"),
    4: dict(density=dict(type="Dehnen", mass=1, scaleRadius=1, gamma=1, axisRatioY=0.8, axisRatioZ=0.6),
            lmax=6, mmax=0, gridSizeR=50, rmin=1e-3, rmax=1e3, symmetry="axisymmetric"),
    5: dict(density=[dict(type="Spheroid", mass=1, scaleRadius=1, gamma=1, beta=4, axisRatioZ=0.6),
                     dict(type="Disk", mass=0.05, scaleRadius=3, scaleHeight=0.3)],
            lmax=12, gridSizeR=80, symmetry="axisymmetric"),
}

SEEDS = {"points1": 1, "orbits1": 2, "particles2": 3, "orbits3": 4, "particles4": 5, "orbits5": 6}


def _isotropic(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1)[:, None]


def dehnen_positions(n, gamma, q=(1.0, 1.0), a=1.0, seed=1):
    """positions from an ellipsoidal Dehnen density: exact inverse of the enclosed-mass
    fraction m(r) = (r/(r+a))^(3-gamma), isotropic direction, then y *= q[0], z *= q[1]"""
    rng = np.random.Generator(np.random.PCG64(seed))
    u = rng.uniform(size=n) ** (1.0 / (3.0 - gamma))
    r = a * u / (1.0 - u)
    x = _isotropic(rng, n) * r[:, None]
    x[:, 1] *= q[0]
    x[:, 2] *= q[1]
    return x


def orbit_ics(positions, potential_fn, seed, umin=0.2, umax=0.8):
    """velocities |v| = u sqrt(-2 Phi(x)), u ~ U[umin, umax], isotropic directions"""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = len(positions)
    vesc = np.sqrt(-2.0 * potential_fn(positions))
    u = rng.uniform(umin, umax, size=n)
    v = _isotropic(rng, n) * (u * vesc)[:, None]
    return np.hstack([positions, v])


def disk_particles(n, vcirc_fn, seed=3, Rd=3.0, hz=0.3, sigma_frac=0.1):
    """disk-like phase-space points: R ~ Gamma(2, Rd) (exponential surface density),
    z = hz artanh(2u-1) (sech^2 profile), phi ~ U[0, 2pi), v_phi = v_circ(R) U[0.8, 1.0],
    v_R, v_z ~ N(0, (sigma_frac v_circ)^2)"""
    rng = np.random.Generator(np.random.PCG64(seed))
    R = rng.gamma(2.0, Rd, size=n)
    z = hz * np.arctanh(2.0 * rng.uniform(size=n) - 1.0)
    phi = rng.uniform(0, 2 * np.pi, size=n)
    vc = vcirc_fn(R)
    vphi = vc * rng.uniform(0.8, 1.0, size=n)
    vR = rng.normal(size=n) * sigma_frac * vc
    vz = rng.normal(size=n) * sigma_frac * vc
    c, s = np.cos(phi), np.sin(phi)
    return np.column_stack([R * c, R * s, z, vR * c - vphi * s, vR * s + vphi * c, vz])


def vcirc_from_force(force_fn):
    """v_circ(R) = sqrt(R dPhi/dR) in the equatorial plane (along x)"""
    def vc(R):
        pts = np.column_stack([R, np.zeros_like(R), np.zeros_like(R)])
        return np.sqrt(-R * force_fn(pts)[:, 0])
    return vc


def equatorial_average(fn, R, nphi=16):
    """azimuthal average over nphi angles in the equatorial plane of fn(points) -> (n, k) or (n,):
    the m = 0 part exactly for harmonics m < nphi (the "axisymmetrized" potential of the
    reference's R_circ / v_circ, src/potential_utils.cpp:608-619)"""
    phi = (np.arange(nphi) + 0.5) * (2 * np.pi / nphi)
    c, s = np.cos(phi), np.sin(phi)
    pts = np.stack([R[:, None] * c, R[:, None] * s, np.zeros((len(R), nphi))], axis=-1).reshape(-1, 3)
    v = np.asarray(fn(pts))
    if v.ndim == 2:   # radial component of a vector field
        v = (v.reshape(len(R), nphi, 3)[:, :, :2] * np.stack([c, s], axis=-1)[None]).sum(-1)
        return v.mean(axis=1)
    return v.reshape(len(R), nphi).mean(axis=1)


def tcirc(potential_fn, force_fn, E, nphi=16, nodes=8193):
    """T_circ(E) = 2 pi R_circ / v_circ(R_circ) of the axisymmetrized potential (the definition of
    T_circ, src/potential_utils.h:83-87): E_c(R) = Phi(R) + R dPhi/dR / 2 and T_c(R) on a grid of
    `nodes` radii log-spaced over [1e-8, 1e8] (spacing 0.0045 in ln R), then ln T_c as a monotone
    cubic (PCHIP) function of E_c, evaluated at E (relative accuracy ~1e-9, far below what an
    integration time of "10 or 100 T_circ" needs; the cost does not grow with the number of E
    values).  E beyond the ends of the grid takes the end value."""
    from scipy.interpolate import PchipInterpolator
    lnR = np.linspace(np.log(1e-8), np.log(1e8), nodes)
    R = np.exp(lnR)
    phi = equatorial_average(potential_fn, R, nphi)
    fR = equatorial_average(force_fn, R, nphi)
    Ec = phi - 0.5 * R * fR
    Tc = 2 * np.pi * R / np.sqrt(np.maximum(-R * fR, 1e-300))
    fin = np.isfinite(Ec) & np.isfinite(Tc)
    Ec, lnT = Ec[fin], np.log(Tc[fin])
    top = np.maximum.accumulate(Ec)
    keep = np.concatenate([[True], Ec[1:] > top[:-1]])     # the nodes where E_c rises strictly
    Ec, lnT = Ec[keep], lnT[keep]
    E = np.asarray(E, dtype=np.float64)
    return np.exp(PchipInterpolator(Ec, lnT, extrapolate=False)(np.clip(E, Ec[0], Ec[-1])))


def orbit_workload(cfg, potential_fn, force_fn, n=None):
    """initial conditions and integration times of the orbit configurations:
    1: 1e4 orbits from the config-1 points, T = 10 T_circ(E);
    3: 1e5 orbits, T = T_circ(E) 10^U[1, 3] (10-1000 dynamical times), Omega = 0.05;
    5: 1e6 orbits, T = 100 T_circ(E)"""
    if cfg == 1:
        n = n or 10000
        pos = dehnen_positions(n, 1.0, q=(0.8, 0.6), seed=SEEDS["points1"])
        ic = orbit_ics(pos, potential_fn, seed=SEEDS["orbits1"])
        scale = np.full(n, 10.0)
    elif cfg == 3:
        n = n or 100000
        pos = dehnen_positions(n, 0.5, q=(0.7, 0.5), seed=SEEDS["orbits3"])
        ic = orbit_ics(pos, potential_fn, seed=SEEDS["orbits3"] + 100)
        rng = np.random.Generator(np.random.PCG64(SEEDS["orbits3"] + 200))
        scale = 10 ** rng.uniform(1, 3, size=n)
    elif cfg == 5:
        n = n or 1000000
        pos = dehnen_positions(n, 1.0, q=(1.0, 0.6), seed=SEEDS["orbits5"])
        ic = orbit_ics(pos, potential_fn, seed=SEEDS["orbits5"] + 100)
        scale = np.full(n, 100.0)
    else:
        raise ValueError("no orbit workload for config %d" % cfg)
    E = potential_fn(ic[:, :3]) + 0.5 * np.sum(ic[:, 3:] ** 2, axis=1)
    T = scale * tcirc(potential_fn, force_fn, E)
    return ic, T
