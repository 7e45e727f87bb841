"""Parity of the device DOP853 orbit integration with the reference's OrbitIntegrator<Car>
(golden vectors from tests/golden/make_golden.py; accuracy 1e-8 as in the benchmark).

Bounds (from the engine's specification):
  * regular orbits: final positions and velocities agree to 1e-7 relative (vector norms);
  * chaotic orbits (a 1e-12 perturbation of the initial point already changes the reference's
    own end point by >1e-9): only the conservation of the (Jacobi) energy is compared --
    the engine's drift must be no worse than 10x the reference's (or 1e-9);
  * accepted step counts of regular orbits agree within 2% (+-2 steps);
  * T = 0 returns the initial point unchanged; the step limit stops orbits with status 1.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def jacobi_energy(pot, w, Omega):
    phi = pot.potential(w[:, :3])
    return phi + 0.5 * np.sum(w[:, 3:] ** 2, axis=1) - Omega * (w[:, 0] * w[:, 4] - w[:, 1] * w[:, 3])


def rel_vec(a, b):
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)


# orbit sets and the evaluator kind of their potential: cfg1, cfg3 (triaxial, <= 8 harmonics in
# registers), cfg3long (config 3 with 10-1000 dynamical times), cfg5 (axisymmetric, lmax 12),
# lop (11 harmonics incl. m < 0: the general kind)
ORBIT_SETS = ["cfg1", "cfg3", "cfg3long", "cfg5", "lop"]
LANE_CASES = [(True, 0), (False, 1), (True, 1), (True, 2), (True, 4), (True, 8), (False, 4)]


def _orbit_cases():
    for cfg in ORBIT_SETS:
        for queue, lanes in LANE_CASES:
            # lane groups serve the multi-harmonic kind only: the other sets run the queue and the
            # one-orbit-per-thread mappings
            if cfg in ("cfg5", "lop") and lanes not in (0, 1):
                continue
            yield cfg, queue, lanes


@pytest.mark.parametrize("cfg,queue,lanes", list(_orbit_cases()))
def test_orbit_parity(cfg, queue, lanes):
    """lanes: lanes of a warp per orbit (0: the autotuner's choice)"""
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "orbits_%s.npz" % cfg))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, cfg.replace("long", "") + ".coef"))
    Omega = float(g["Omega"])
    agama_b200.set_orbit_lanes(lanes)
    try:
        final, info = agama_b200.orbit(pot, g["ic"], g["T"], Omega=Omega, accuracy=float(g["accuracy"]),
                                       queue=queue, info=True)
    finally:
        agama_b200.set_orbit_lanes(0)
    reg = g["regular"] & (g["status"] == 0)
    assert np.all(info["status"] == g["status"])
    epos = rel_vec(final[reg, :3], g["final"][reg, :3])
    evel = rel_vec(final[reg, 3:], g["final"][reg, 3:])
    assert epos.max() <= 1e-7 and evel.max() <= 1e-7, (epos.max(), evel.max())
    s, sr = info["steps"][reg], g["steps"][reg]
    assert np.all(np.abs(s - sr) <= np.maximum(2, 0.02 * sr)), np.abs(s - sr).max()
    # energy conservation: per orbit for the regular ones; for the chaotic ones (whose drift over
    # hundreds of periods is a random walk of the integration errors, different on both sides) the
    # median and the largest drift of the set
    E0 = jacobi_energy(pot, g["ic"], Omega)
    drift = np.abs(jacobi_energy(pot, final, Omega) / E0 - 1)
    drift_ref = np.abs(jacobi_energy(pot, g["final"], Omega) / E0 - 1)
    assert np.all(drift[reg] <= np.maximum(10 * drift_ref[reg], 1e-9)), (drift[reg].max(), drift_ref[reg].max())
    ok = g["status"] == 0
    assert np.median(drift[ok]) <= np.maximum(10 * np.median(drift_ref[ok]), 1e-9), (np.median(drift[ok]),
                                                                                  np.median(drift_ref[ok]))
    assert drift[ok].max() <= np.maximum(10 * drift_ref[ok].max(), 1e-9), (drift[ok].max(), drift_ref[ok].max())


@pytest.mark.parametrize("cfg", ["cfg1", "cfg3", "cfg5"])
def test_orbit_bits_independent_of_launch_shape(cfg):
    """every lane count and block size gives the same bits (the harmonics of a lane group are
    summed in one order; the block only groups orbits), so the autotuner's timing-based choice
    never changes a result"""
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "orbits_%s.npz" % cfg))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, cfg + ".coef"))
    results = []
    lane_counts = (1, 2, 4, 8) if cfg != "cfg5" else (1,)
    for lanes in lane_counts:
        for block in (32, 64, 128):
            agama_b200.set_orbit_lanes(lanes)
            agama_b200.set_orbit_block(block)
            try:
                results.append(agama_b200.orbit(pot, g["ic"], g["T"], Omega=float(g["Omega"]),
                                                accuracy=float(g["accuracy"]), info=True))
            finally:
                agama_b200.set_orbit_lanes(0)
                agama_b200.set_orbit_block(0)
    for final, info in results[1:]:
        assert np.array_equal(final, results[0][0])
        assert np.array_equal(info["steps"], results[0][1]["steps"])


def test_orbit_edge_cases():
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "orbits_cfg1.npz"))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg1.coef"))
    # zero integration time: the initial point comes back unchanged
    i0 = int(np.where(g["T"] == 0)[0][0])
    f, info = agama_b200.orbit(pot, g["ic"][i0:i0 + 1], 0.0, info=True)
    assert np.array_equal(f[0], g["ic"][i0]) and info["steps"][0] == 0
    # step limit: status 1 after exactly 10 steps, near the reference's point after 10 steps.
    # (The end time of an intermediate step is set by the step-size controller, whose error norm
    # is a difference of stage combinations that cancel to O(h^8): the step lengths agree only to
    # ~1e-9 relative, so the point after 10 steps is compared loosely; full integrations end at
    # exactly T and are held to 1e-7 above.)
    f, info = agama_b200.orbit(pot, g["ic"][:4], g["T"][:4], maxNumSteps=10, info=True)
    assert np.all(info["status"] == g["status_maxsteps10"]) and np.all(info["steps"] == g["steps_maxsteps10"])
    assert rel_vec(f[:, :3], g["final_maxsteps10"][:, :3]).max() <= 1e-5
    # empty batch
    assert agama_b200.orbit(pot, np.zeros((0, 6)), 1.0).shape == (0, 6)


def test_orbit_device_pointers():
    import torch
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "orbits_cfg1.npz"))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg1.coef"))
    ic = torch.tensor(g["ic"], device="cuda")
    T = torch.tensor(g["T"], device="cuda")
    out, info = agama_b200.orbit(pot, ic, T, info=True)
    torch.cuda.synchronize()
    host = agama_b200.orbit(pot, g["ic"], g["T"])
    assert np.array_equal(out.cpu().numpy(), host)


@pytest.mark.parametrize("cfg", ["cfg1", "cfg3"])
def test_trajectory_samples(cfg):
    """samples at 11 regular times from the dense output of the steps against the reference's
    RuntimeTrajectory: regular orbits to 1e-7 (positions and velocities), NaN pattern identical
    (the zero-time orbit: its start as samples 0 and 1), the last sample the final point"""
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "orbits_%s.npz" % cfg))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, cfg + ".coef"))
    Omega = float(g["Omega"])
    times, traj = agama_b200.trajectory(pot, g["ic"], g["T"], 11, Omega=Omega, accuracy=float(g["accuracy"]))
    ref = g["traj11"]
    assert np.array_equal(np.isnan(traj), np.isnan(ref))
    reg = g["regular"] & (g["status"] == 0)
    for k in range(11):
        ok = reg & np.all(np.isfinite(ref[:, k]), axis=1)
        epos = rel_vec(traj[ok, k, :3], ref[ok, k, :3])
        evel = rel_vec(traj[ok, k, 3:], ref[ok, k, 3:])
        assert epos.max(initial=0) <= 1e-7 and evel.max(initial=0) <= 1e-7, (k, epos.max(), evel.max())
    final = agama_b200.orbit(pot, g["ic"], g["T"], Omega=Omega, accuracy=float(g["accuracy"]))
    fin = g["T"] != 0
    assert np.allclose(traj[fin, -1], final[fin], rtol=1e-12, atol=1e-12 * np.max(np.abs(final[fin])))


def test_orbit_graph_replays_and_continues():
    """a captured orbit batch: one launch equals the direct call bit for bit; with the end points
    written over the starts, two launches of T continue the orbits: bit for bit the same as two
    direct calls, the second started from the end of the first (a restart, as the reference's
    integrator started again from a point)"""
    import torch
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "orbits_cfg1.npz"))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg1.coef"))
    ok = g["T"] > 0
    ic = torch.tensor(g["ic"][ok], device="cuda")
    T = torch.tensor(g["T"][ok], device="cuda")
    direct = agama_b200.orbit(pot, ic, T)
    graph = agama_b200.OrbitGraph(pot, ic, T)
    assert graph.lanes in (1, 2, 4, 8) and graph.block in (32, 64, 128)
    once = graph.launch()
    torch.cuda.synchronize()
    assert torch.equal(once, direct)
    x = ic.clone()
    seg = agama_b200.OrbitGraph(pot, x, T, final=x)
    seg.launch()
    seg.launch()
    twice = agama_b200.orbit(pot, agama_b200.orbit(pot, ic, T), T)
    torch.cuda.synchronize()
    assert torch.equal(x, twice)


@pytest.mark.parametrize("cfg", ["cfg1", "cfg3"])
def test_orbit_mixed_precision(cfg):
    """FP32 non-axisymmetric harmonics: final points of regular orbits within 1e-3 relative of the
    reference's (FP64 is held to 1e-7; measured on B200: 1.5e-4 for config 1's orbits of 10
    circular periods, 3.6e-5 for config 3's), and the per-orbit error statement (Jacobi energy)
    within 1e-5 for regular orbits; over all orbits (chaotic ones drift in either precision) the
    median within 3x and the largest within 10x the FP64 run's (measured on config 3: largest
    1.8e-5 against 5.7e-6): the FP32 rounding of the m != 0 force shifts the orbital phases, which
    grows linearly with the integration time"""
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "orbits_%s.npz" % cfg))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, cfg + ".coef"))
    Omega = float(g["Omega"])
    agama_b200.set_orbit_precision(True)
    try:
        final, info = agama_b200.orbit(pot, g["ic"], g["T"], Omega=Omega, accuracy=float(g["accuracy"]), info=True)
    finally:
        agama_b200.set_orbit_precision(False)
    final64 = agama_b200.orbit(pot, g["ic"], g["T"], Omega=Omega, accuracy=float(g["accuracy"]))
    assert not np.array_equal(final, final64)          # the FP32 path did run
    reg = g["regular"] & (g["status"] == 0)
    assert np.all(info["status"] == g["status"])
    epos = rel_vec(final[reg, :3], g["final"][reg, :3])
    evel = rel_vec(final[reg, 3:], g["final"][reg, 3:])
    ok = g["status"] == 0
    err = agama_b200.jacobi_energy_error(pot, g["ic"][ok], final[ok], Omega)
    err64 = agama_b200.jacobi_energy_error(pot, g["ic"][ok], final64[ok], Omega)
    print(cfg, "mixed vs reference: pos %.3g vel %.3g; Jacobi energy error mixed %.3g fp64 %.3g" %
          (epos.max(), evel.max(), err.max(), err64.max()))
    assert epos.max() <= 1e-3 and evel.max() <= 1e-3, (epos.max(), evel.max())
    # regular orbits: 1e-5; all orbits (chaotic ones drift in either precision): the distribution
    # of the errors against FP64's
    assert err[reg[ok]].max() <= 1e-5, err[reg[ok]].max()
    assert np.median(err) <= 3 * np.median(err64) + 1e-8, (np.median(err), np.median(err64))
    assert err.max() <= 10 * err64.max() + 1e-6, (err.max(), err64.max())
    # the setting is off again: FP64 results are the reference's to 1e-7
    again = agama_b200.orbit(pot, g["ic"], g["T"], Omega=Omega, accuracy=float(g["accuracy"]))
    assert np.array_equal(again, final64)
