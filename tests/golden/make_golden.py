"""Generate the golden fixtures of the parity tests from the reference implementation.

Run here, where the reference sources exist and the oracle has been built (make -C oracle):

    python tests/golden/make_golden.py [potentials|orbits|actions|utils|all]

It writes, into tests/golden/:
  <name>.coef            Multipole coefficient files written by the reference (writePotential)
                         for the benchmark potentials and a few extra cases (1-D path, spherical);
  potential_<name>.npz   evaluation points (incl. edge cases) with the reference's potential,
                         gradient and Hessian at them;
  orbits_<name>.npz      initial conditions, integration times and the reference's final
                         phase-space points, accepted step counts and statuses (configs 1, 3 and 5,
                         the general-kind potential 'lop', long config-3 times 'cfg3long');
  actions_<name>.npz     phase-space points with the reference's Staeckel-fudge actions (fixed
                         focal distance and through ActionFinderAxisymFudge), plus the finder's
                         focal-distance table and L_circ(E) spline;
  target_<name>.npz      the reference's density-grid targets (runtime functions) of the golden
                         orbits (configs 1 and 3);
  utils_<name>.npz       density at the potential_<name> points and R_circ(E), R_max(E),
                         R_from_Lz(L), peri/apocentre radii of (E, L), through the reference's
                         plain-C interface.
All inputs are synthetic and seeded (agama_b200/workloads.py); no external dataset is involved.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))

from agama_b200 import workloads  # noqa: E402
from oracle import ref  # noqa: E402

# extra potentials exercising the other evaluation paths
EXTRA_POTENTIALS = {
    # lmax <= 2: per-(l,m) 1-D splines with the closed-form l<=2 transform
    "quad": dict(density=dict(type="Dehnen", mass=1, scaleRadius=1, gamma=1.5, axisRatioY=0.7, axisRatioZ=0.5),
                 lmax=2, gridSizeR=30, symmetry="triaxial"),
    # spherical: lmax = 0
    "sph": dict(density=dict(type="Plummer", mass=2, scaleRadius=0.7), lmax=0, gridSizeR=25),
    # odd harmonics and m < 0 terms (no reflection symmetry): general inverse transform
    "lop": dict(density=dict(type="Dehnen", mass=1, scaleRadius=1, gamma=1, axisRatioY=0.8, axisRatioZ=0.6,
                             orientation=[0.3, 0.5, 0.2], center=[0.05, -0.02, 0.03]),
                lmax=5, gridSizeR=40, symmetry="none"),
}


def build_reference_potential(spec):
    """construct a Multipole from a density with the reference's Python interface"""
    import agama
    spec = dict(spec)
    d = spec.pop("density")
    comps = []
    for x in (d if isinstance(d, list) else [d]):
        x = dict(x)
        if x["type"] in ("MiyamotoNagai", "NFW"):
            comps.append(agama.Potential(**x))
        else:
            comps.append(agama.Density(**x))
    dens = comps[0] if len(comps) == 1 else agama.Density(*comps)
    return agama.Potential(type="Multipole", density=dens, **spec)


def coef_path(name):
    return os.path.join(HERE, name + ".coef")


def make_potentials():
    specs = {"cfg%d" % k: v for k, v in workloads.CONFIG_POTENTIALS.items()}
    specs.update(EXTRA_POTENTIALS)
    for name, spec in specs.items():
        pot = build_reference_potential(spec)
        pot.export(coef_path(name))
        print("wrote", coef_path(name))


def eval_points(coef, seed, n=1500):
    """points spanning the inner asymptote, the spline region and the outer asymptote,
    plus edge cases: on the z axis, in the equatorial plane, at the grid radii, near r=0"""
    rng = np.random.Generator(np.random.PCG64(seed))
    with open(coef) as f:
        rows = f.read().split("#Phi")[1].split("\n")[2:]
    radii = np.array([float(r.split("\t")[0]) for r in rows if r.strip() and not r.startswith("#")][:1000])
    radii = radii[: np.argmax(np.diff(radii) <= 0) + 1] if np.any(np.diff(radii) <= 0) else radii
    rmin, rmax = radii[0], radii[-1]
    r = np.exp(rng.uniform(np.log(rmin / 30), np.log(rmax * 30), size=n))
    x = rng.normal(size=(n, 3))
    x *= (r / np.linalg.norm(x, axis=1))[:, None]
    edge = []
    for rr in [rmin * 0.5, rmin, rmin * (1 + 1e-5), radii[1], radii[len(radii) // 2], rmax * (1 - 1e-5), rmax, rmax * 2]:
        edge += [[rr, 0, 0], [0, 0, rr], [0, 0, -rr], [0, rr, 0], [-rr / 2, rr / 2, rr / np.sqrt(2)],
                 [rr * 0.6, -rr * 0.8, 0]]
    edge += [[1e-7, 2e-7, -1e-7], [1e5, -2e5, 3e5], [0.3, 0, 0.4], [-0.3, 0, 0.4], [0, -0.5, 1e-12]]
    return np.vstack([x, np.array(edge, dtype=float)])


def make_potential_vectors():
    names = ["cfg%d" % k for k in workloads.CONFIG_POTENTIALS] + list(EXTRA_POTENTIALS)
    for i, name in enumerate(names):
        pot = ref.Potential(file=coef_path(name))
        pts = eval_points(coef_path(name), seed=100 + i)
        phi, grad, hess = pot.eval(pts, hess=True)
        out = os.path.join(HERE, "potential_%s.npz" % name)
        np.savez_compressed(out, points=pts, phi=phi, grad=grad, hess=hess)
        print("wrote", out, len(pts))


def tcirc(coef, E):
    """T_circ(E) of the reference (potential_utils.h:83-87) through its Python interface"""
    import agama
    return agama.Potential(file=coef).Tcirc(E)


def regular_flags(pot, ic, T, Omega, accuracy=1e-8):
    """an orbit counts as regular when a 1e-12 relative perturbation of its initial point
    changes the final point by less than 1e-9 (relative): no exponential divergence over T"""
    f0, _, _ = pot.orbits(ic, T, Omega=Omega, accuracy=accuracy)
    f1, _, _ = pot.orbits(ic * (1 + 1e-12), T, Omega=Omega, accuracy=accuracy)
    d = np.max(np.abs(f1 - f0) / np.maximum(np.abs(f0), 1e-300), axis=1)
    sc = np.linalg.norm(f1[:, :3] - f0[:, :3], axis=1) / np.linalg.norm(f0[:, :3], axis=1)
    return (sc < 1e-9) & (d < 1e-6)


def make_orbit_vectors():
    # config 1: orbits drawn as in the benchmark, T = 10 T_circ(E)
    coef = coef_path("cfg1")
    pot = ref.Potential(file=coef)
    n = 48
    x = workloads.dehnen_positions(n, gamma=1, q=(0.8, 0.6), seed=workloads.SEEDS["orbits1"])
    ic = workloads.orbit_ics(x, lambda p: pot.eval(p)[0], seed=workloads.SEEDS["orbits1"] + 100)
    E = pot.eval(ic[:, :3])[0] + 0.5 * np.sum(ic[:, 3:] ** 2, axis=1)
    T = 10 * tcirc(coef, E)
    # edge cases: zero time, backward integration, an escaping orbit, a step-limited orbit
    ic = np.vstack([ic, ic[:3], [[0.5, 0.1, 0.2, 3.0, 0.5, -0.2]]])
    T = np.concatenate([T, [0.0, -T[1], T[2], 50.0]])
    final, steps, status = pot.orbits(ic, T, Omega=0.0, accuracy=1e-8)
    fin10, steps10, st10 = pot.orbits(ic[:4], T[:4], Omega=0.0, accuracy=1e-8, maxSteps=10)
    regular = regular_flags(pot, ic, T, 0.0)
    traj = pot.orbits_traj(ic, T, 11, Omega=0.0, accuracy=1e-8)
    np.savez_compressed(os.path.join(HERE, "orbits_cfg1.npz"), ic=ic, T=T, Omega=0.0, accuracy=1e-8,
                        final=final, steps=steps, status=status, regular=regular,
                        final_maxsteps10=fin10, steps_maxsteps10=steps10, status_maxsteps10=st10, traj11=traj)
    print("cfg1 orbits", len(ic), "regular", regular.sum(), "steps", steps.min(), steps.max())
    # config 3: rotating frame Omega = 0.05, uneven times 10^U[1, 1.5] T_circ
    coef = coef_path("cfg3")
    pot = ref.Potential(file=coef)
    n = 24
    x = workloads.dehnen_positions(n, gamma=0.5, q=(0.7, 0.5), seed=workloads.SEEDS["orbits3"])
    ic = workloads.orbit_ics(x, lambda p: pot.eval(p)[0], seed=workloads.SEEDS["orbits3"] + 100)
    E = pot.eval(ic[:, :3])[0] + 0.5 * np.sum(ic[:, 3:] ** 2, axis=1)
    rng = np.random.Generator(np.random.PCG64(41))
    T = tcirc(coef, E) * 10 ** rng.uniform(1, 1.5, size=n)
    final, steps, status = pot.orbits(ic, T, Omega=0.05, accuracy=1e-8)
    regular = regular_flags(pot, ic, T, 0.05)
    traj = pot.orbits_traj(ic, T, 11, Omega=0.05, accuracy=1e-8)
    np.savez_compressed(os.path.join(HERE, "orbits_cfg3.npz"), ic=ic, T=T, Omega=0.05, accuracy=1e-8,
                        final=final, steps=steps, status=status, regular=regular, traj11=traj)
    print("cfg3 orbits", len(ic), "regular", regular.sum(), "steps", steps.min(), steps.max())


def make_more_orbit_vectors():
    """orbit sets for the other evaluator kinds and the long config-3 times:
    orbits_cfg5.npz  the axisymmetric kind (lmax 12, one harmonic): 192 orbits of the config-5
                     workload, T = 100 T_circ(E);
    orbits_lop.npz   the general kind (11 harmonics, m < 0 terms, no symmetry): 48 orbits,
                     T = 10 T_circ(E);
    orbits_cfg3long.npz  480 orbits of the config-3 distribution with T = T_circ(E) 10^U[1, 3]
                     (10-1000 dynamical times) in the frame rotating at Omega = 0.05; only the
                     orbits that the reference finishes within MAX_STEPS_LONG accepted steps are kept
                     (the rest of the workload's tail needs up to 1e7 steps per orbit)."""
    MAX_STEPS_LONG = 40000
    for name, n, scale_fn, Omega in (("cfg5", 192, None, 0.0), ("lop", 48, None, 0.0), ("cfg3", 480, None, 0.05)):
        coef = coef_path(name)
        pot = ref.Potential(file=coef)
        potential_fn = lambda p: pot.eval(p)[0]
        force_fn = lambda p: -pot.eval(p)[1]
        if name == "cfg5":
            ic, T = workloads.orbit_workload(5, potential_fn, force_fn, n)
        elif name == "cfg3":
            ic, T = workloads.orbit_workload(3, potential_fn, force_fn, n)
        else:
            x = workloads.dehnen_positions(n, gamma=1, q=(0.8, 0.6), seed=707)
            ic = workloads.orbit_ics(x, potential_fn, seed=708)
            E = potential_fn(ic[:, :3]) + 0.5 * np.sum(ic[:, 3:] ** 2, axis=1)
            T = 10 * workloads.tcirc(potential_fn, force_fn, E)
        mx = MAX_STEPS_LONG if name == "cfg3" else 0
        final, steps, status = pot.orbits(ic, T, Omega=Omega, accuracy=1e-8, maxSteps=mx)
        if name == "cfg3":
            keep = status == 0
            ic, T, final, steps, status = ic[keep], T[keep], final[keep], steps[keep], status[keep]
        f1, _, _ = pot.orbits(ic * (1 + 1e-12), T, Omega=Omega, accuracy=1e-8, maxSteps=mx)
        d = np.max(np.abs(f1 - final) / np.maximum(np.abs(final), 1e-300), axis=1)
        sc = np.linalg.norm(f1[:, :3] - final[:, :3], axis=1) / np.linalg.norm(final[:, :3], axis=1)
        regular = (sc < 1e-9) & (d < 1e-6)
        fname = "orbits_%s.npz" % ("cfg3long" if name == "cfg3" else name)
        np.savez_compressed(os.path.join(HERE, fname), ic=ic, T=T, Omega=Omega, accuracy=1e-8,
                            final=final, steps=steps, status=status, regular=regular)
        print(fname, len(ic), "regular", regular.sum(), "steps", steps.min(), steps.max(),
              "T/T_circ max", "%.0f" % (T / workloads.tcirc(potential_fn, force_fn,
                                                            potential_fn(ic[:, :3]) + 0.5 * np.sum(ic[:, 3:] ** 2, 1))).max())


def make_target_vectors():
    """runtime functions of orbits: the reference's orbit(..., targets=[Target(...)]) (its
    RuntimeFncTarget with TargetDensityClassic) on the config-1 and config-3 golden orbits:
    target_<name>.npz holds the grid parameters and the float32 matrices (orbits x cells)"""
    import agama
    for name, grids in (("cfg1", [("DensityClassicTopHat", 2, 0.8, 0.6), ("DensityClassicLinear", 3, 1.0, 1.0)]),
                        ("cfg3", [("DensityClassicTopHat", 3, 0.7, 0.5)])):
        g = np.load(os.path.join(HERE, "orbits_%s.npz" % name))
        pot = agama.Potential(file=coef_path(name))
        gridr = np.array([0, 0.1, 0.25, 0.5, 1, 2, 4, 8, 16.0])
        out = dict(ic=g["ic"], T=g["T"], Omega=g["Omega"], accuracy=g["accuracy"], gridr=gridr)
        for k, (typ, strips, qy, qz) in enumerate(grids):
            t = agama.Target(type=typ, gridr=gridr, stripsPerPane=strips, axisRatioY=qy, axisRatioZ=qz)
            m = agama.orbit(potential=pot, ic=g["ic"], time=g["T"], Omega=float(g["Omega"]), targets=[t],
                            accuracy=float(g["accuracy"]))
            out["type%d" % k] = typ
            out["strips%d" % k] = strips
            out["axes%d" % k] = np.array([qy, qz])
            out["result%d" % k] = np.asarray(m)
            print(name, typ, np.asarray(m).shape)
        np.savez_compressed(os.path.join(HERE, "target_%s.npz" % name), **out)


def action_points(pot, n, seed, Rd=3.0, hz=0.3):
    """disk-like points of the benchmark distribution plus edge cases: in the plane (z = 0),
    no rotation (Lz = 0), counter-rotating, nearly circular, on the z axis, unbound"""
    vc = workloads.vcirc_from_force(lambda p: -pot.eval(p)[1])
    w = workloads.disk_particles(n, vc, seed=seed, Rd=Rd, hz=hz)
    v1 = float(vc(np.array([1.0]))[0])
    v5 = float(vc(np.array([5.0]))[0])
    edge = np.array([
        [2.0, 0.0, 0.0, 0.05, v1 * 0.9, 0.03],      # in the equatorial plane
        [3.0, 0.0, 0.4, 0.1, 0.0, 0.05],            # Lz = 0
        [-4.0, 1.0, -0.3, 0.02, -0.1, 0.01],        # counter-rotating (Lz < 0)
        [5.0, 0.0, 0.0, 0.0, v5, 0.0],              # circular orbit in the plane
        [5.0, 0.0, 0.0, 0.0, v5, 1e-6],             # nearly circular
        [0.0, 0.0, 1.5, 0.1, 0.05, 0.02],           # on the z axis
        [1.0, 0.5, 0.2, 3.0, 2.0, 1.0],             # unbound (E > 0)
        [8.0, -2.0, 3.0, -0.05, 0.1, 0.12],         # thick, eccentric
    ])
    return np.vstack([w, edge])


def make_action_vectors():
    for name, n, seed in [("cfg2", 2000, 303), ("cfg5", 600, 606), ("cfg4", 600, 505)]:
        coef = coef_path(name)
        pot = ref.Potential(file=coef)
        pts = action_points(pot, n, seed)
        af = ref.ActionFinder(pot)
        af.evalcount(reset=True)
        act_af, fd = af.actions(pts, with_fd=True)
        evals_per_point = af.evalcount(reset=True) / len(pts)
        act_fd, counts = pot.actions_fd(pts, fd, count=True)
        _, ang_fd, freq_fd = pot.actions_angles_fd(pts, fd)
        tab = af.tables()
        np.savez_compressed(os.path.join(HERE, "actions_%s.npz" % name), points=pts, fd=fd,
                            act_finder=act_af, act_fd=act_fd, evals_fd=counts, ang_fd=ang_fd, freq_fd=freq_fd,
                            evals_per_point_finder=evals_per_point, **{"tab_" + k: v for k, v in tab.items()})
        print(name, "actions", len(pts), "evals/point %.1f" % evals_per_point,
              "table", tab["delta"].shape, "LofE", tab["lofe"].shape)


def make_utility_vectors():
    """density and the radius routines through the reference's plain-C interface
    (agama_evalDensity, agama_R_circ, agama_R_from_Lz, agama_R_max, agama_findPlanarOrbitExtent)"""
    for i, name in enumerate(["cfg1", "cfg2", "quad", "sph", "lop"]):
        cpot = ref.CInterfacePotential("file=" + coef_path(name))
        pot = ref.Potential(file=coef_path(name))
        pts = np.load(os.path.join(HERE, "potential_%s.npz" % name))["points"]
        rho = cpot.density(pts)
        rng = np.random.Generator(np.random.PCG64(900 + i))
        # energies of radii log-uniform over [1e-4, 1e4] (inside, between and beyond the grid ends)
        r = 10 ** rng.uniform(-4, 4, size=120)
        E = pot.eval(np.column_stack([r, 0 * r, 0 * r]))[0]
        phi0 = pot.eval(np.zeros((1, 3)))[0][0]
        E = np.concatenate([E, [phi0 * 1.000001, 0.5 * phi0, -1e-12, 0.0, 0.1]])
        # angular momenta log-uniform, with zero and a negative value
        L = np.concatenate([10 ** rng.uniform(-4, 3, size=120), [0.0, -0.7, 1e-8]])
        # (E, L) pairs: L a fraction u of the circular value at E (radial, eccentric, nearly
        # circular, above circular) and energies outside the allowed range
        rr = 10 ** rng.uniform(-3.5, 3.5, size=100)
        Ep = pot.eval(np.column_stack([rr, 0 * rr, 0 * rr]))[0]
        Rc = cpot.R_circ(Ep)
        g = pot.eval(np.column_stack([Rc, 0 * Rc, 0 * Rc]))[1]
        Lc = Rc * np.sqrt(np.abs(Rc * g[:, 0]))
        u = np.concatenate([rng.uniform(0, 1, size=90), [0.0, 0.9999995, 0.999999, 1.0, 1.05, 0.5, 0.3, 0.1,
                                                        0.99, 1e-6]])
        EL = np.column_stack([Ep, u * Lc])
        EL = np.vstack([EL, [[phi0 * 1.01, 0.1], [0.1, 0.5]]])
        np.savez_compressed(os.path.join(HERE, "utils_%s.npz" % name), points=pts, rho=rho, E=E,
                            Rcirc=cpot.R_circ(E), Rmax=cpot.R_max(E), L=L, RfromLz=cpot.R_from_Lz(L),
                            EL=EL, periapo=cpot.periapo(EL[:, 0], EL[:, 1]))
        print(name, "density points", len(pts), "energies", len(E), "L", len(L), "(E,L)", len(EL))


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("potentials", "all"):
        make_potentials()
        make_potential_vectors()
    if what in ("orbits", "all"):
        make_orbit_vectors()
    if what in ("orbits", "more_orbits", "all"):
        make_more_orbit_vectors()
    if what in ("targets", "all"):
        make_target_vectors()
    if what in ("actions", "all"):
        make_action_vectors()
    if what in ("utils", "all"):
        make_utility_vectors()
