"""CPU checks of the oracles themselves (no GPU).

1. The reference built from its own sources (oracle/_ref) reproduces the committed golden vectors
   on samples of their inputs: Multipole evaluation, DOP853 orbits, Staeckel-fudge actions (fixed
   focal distance and through its ActionFinderAxisymFudge) and the plain-C interface's density and
   radius routines.  This pins the fixtures to the oracle build (same compiler, flags and GSL
   stand-in) that the GPU parity tests compare against.
2. The FP64 restatement of the bracket-predictor network (oracle/mlp_ref.py), the gradient oracle
   of the tensor-core training kernels, against central finite differences of its own loss."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

ref = pytest.importorskip("oracle.ref")
needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built (needs the reference sources)")


@needs_ref
@pytest.mark.parametrize("name", ["cfg1", "cfg2", "quad", "sph", "lop"])
def test_reference_potential_reproduces_golden(name):
    g = np.load(os.path.join(GOLDEN, "potential_%s.npz" % name))
    pot = ref.Potential(file=os.path.join(GOLDEN, name + ".coef"))
    k = np.arange(0, len(g["points"]), 7)
    phi, grad, hess = pot.eval(g["points"][k], hess=True, nthreads=1)
    np.testing.assert_array_equal(phi, g["phi"][k])
    np.testing.assert_array_equal(grad, g["grad"][k])
    np.testing.assert_array_equal(hess, g["hess"][k])


@needs_ref
def test_reference_orbits_reproduce_golden():
    g = np.load(os.path.join(GOLDEN, "orbits_cfg1.npz"))
    pot = ref.Potential(file=os.path.join(GOLDEN, "cfg1.coef"))
    final, steps, status = pot.orbits(g["ic"][:6], g["T"][:6], Omega=float(g["Omega"]),
                                      accuracy=float(g["accuracy"]), nthreads=1)
    np.testing.assert_array_equal(final, g["final"][:6])
    np.testing.assert_array_equal(steps, g["steps"][:6])
    np.testing.assert_array_equal(status, g["status"][:6])


@needs_ref
@pytest.mark.parametrize("name", ["cfg5", "lop", "cfg3long"])
def test_reference_orbit_sets_reproduce_golden(name):
    """the axisymmetric (config 5), general-kind and long config-3 orbit sets"""
    g = np.load(os.path.join(GOLDEN, "orbits_%s.npz" % name))
    pot = ref.Potential(file=os.path.join(GOLDEN, name.replace("long", "") + ".coef"))
    k = np.arange(0, len(g["ic"]), max(1, len(g["ic"]) // 6))[:6]
    final, steps, status = pot.orbits(g["ic"][k], g["T"][k], Omega=float(g["Omega"]),
                                      accuracy=float(g["accuracy"]), nthreads=1)
    np.testing.assert_array_equal(final, g["final"][k])
    np.testing.assert_array_equal(steps, g["steps"][k])
    np.testing.assert_array_equal(status, g["status"][k])


@needs_ref
def test_reference_rotating_frame_and_trajectories_reproduce_golden():
    g = np.load(os.path.join(GOLDEN, "orbits_cfg3.npz"))
    pot = ref.Potential(file=os.path.join(GOLDEN, "cfg3.coef"))
    final, steps, _ = pot.orbits(g["ic"][:3], g["T"][:3], Omega=float(g["Omega"]), accuracy=float(g["accuracy"]),
                                 nthreads=1)
    np.testing.assert_array_equal(final, g["final"][:3])
    np.testing.assert_array_equal(steps, g["steps"][:3])
    traj = pot.orbits_traj(g["ic"][:3], g["T"][:3], 11, Omega=float(g["Omega"]), accuracy=float(g["accuracy"]),
                           nthreads=1)
    np.testing.assert_array_equal(traj, g["traj11"][:3])


@needs_ref
def test_reference_targets_reproduce_golden():
    """the reference's orbit(..., targets=[Target]) through its own Python module built here"""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(ref.__file__), "_ref"))
    import agama
    g = np.load(os.path.join(GOLDEN, "target_cfg1.npz"))
    pot = agama.Potential(file=os.path.join(GOLDEN, "cfg1.coef"))
    qy, qz = g["axes0"]
    t = agama.Target(type=str(g["type0"]), gridr=g["gridr"], stripsPerPane=int(g["strips0"]), axisRatioY=qy,
                     axisRatioZ=qz)
    m = agama.orbit(potential=pot, ic=g["ic"][:4], time=g["T"][:4], targets=[t], accuracy=float(g["accuracy"]))
    np.testing.assert_array_equal(np.asarray(m), g["result0"][:4])


@needs_ref
def test_reference_angles_reproduce_golden():
    g = np.load(os.path.join(GOLDEN, "actions_cfg5.npz"))
    pot = ref.Potential(file=os.path.join(GOLDEN, "cfg5.coef"))
    act, ang, freq = pot.actions_angles_fd(g["points"][:100], g["fd"][:100], nthreads=1)
    np.testing.assert_array_equal(ang, g["ang_fd"][:100])
    np.testing.assert_array_equal(freq, g["freq_fd"][:100])


@needs_ref
def test_reference_actions_reproduce_golden():
    g = np.load(os.path.join(GOLDEN, "actions_cfg2.npz"))
    pot = ref.Potential(file=os.path.join(GOLDEN, "cfg2.coef"))
    pts, fd = g["points"][:300], g["fd"][:300]
    np.testing.assert_array_equal(pot.actions_fd(pts, fd, nthreads=1), g["act_fd"][:300])
    af = ref.ActionFinder(pot)
    J, fd2 = af.actions(pts, nthreads=1, with_fd=True)
    np.testing.assert_array_equal(J, g["act_finder"][:300])
    np.testing.assert_array_equal(fd2, fd)


@needs_ref
@pytest.mark.parametrize("name", ["cfg1", "cfg2", "lop"])
def test_reference_c_interface_reproduces_golden(name):
    g = np.load(os.path.join(GOLDEN, "utils_%s.npz" % name))
    cpot = ref.CInterfacePotential("file=" + os.path.join(GOLDEN, name + ".coef"))
    k = np.arange(0, len(g["points"]), 25)
    np.testing.assert_array_equal(cpot.density(g["points"][k]), g["rho"][k])
    np.testing.assert_array_equal(cpot.R_circ(g["E"]), g["Rcirc"])
    np.testing.assert_array_equal(cpot.R_max(g["E"]), g["Rmax"])
    np.testing.assert_array_equal(cpot.R_from_Lz(g["L"]), g["RfromLz"])
    np.testing.assert_array_equal(cpot.periapo(g["EL"][:, 0], g["EL"][:, 1]), g["periapo"])


def test_network_oracle_gradient_matches_finite_differences():
    from oracle import mlp_ref
    rng = np.random.default_rng(7)
    n = mlp_ref.num_params()
    p = rng.normal(0, 0.2, n)
    x = rng.normal(0, 1, (16, 6))
    t = rng.uniform(0, 1, (16, 3))
    m = (rng.uniform(0, 1, (16, 3)) > 0.2).astype(float)
    _, grad = mlp_ref.loss_grad(p, x, t, m)          # FP64 (no BF16 rounding): exact gradient
    for j in rng.choice(n, 40, replace=False):
        h = 1e-6
        e = np.zeros(n)
        e[j] = h
        fd = (mlp_ref.loss_grad(p + e, x, t, m)[0] - mlp_ref.loss_grad(p - e, x, t, m)[0]) / (2 * h)
        assert abs(fd - grad[j]) <= 1e-7 * max(1.0, abs(grad[j])) + 1e-9, (j, fd, grad[j])
