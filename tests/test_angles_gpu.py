"""Angles and frequencies of the Staeckel fudge against the reference (golden vectors from
tests/golden/make_golden.py: actions::evalAxisymFudge with angles and frequencies, given focal
distances).  The engine evaluates the same integrals on the same Gauss-Legendre nodes, so the
bound is the action bound: 1e-6 relative for frequencies (with 1e-9 of the largest frequency of
the point for components that vanish), and 1e-6 radian for angles (compared modulo 2 pi).

Excluded: orbits whose radial action is below 1e-7 of the total (a circular orbit and a nearly
circular one among the edge cases).  Their radial turning points lie at the round-off level of
F(lambda), so whether an orbit counts as a shell orbit (and gets the limiting value of the
integrals) or has a round-off-sized radial range is decided by the last bits of the potential,
in the reference as here: the reference itself gives Omega_r = 0.041 for the circular orbit and
0.161 for the one with v_z = 1e-6."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CFGS = ["cfg2", "cfg5", "cfg4"]


def well_conditioned(Jref):
    """points whose radial and vertical motions are not at the round-off level"""
    tot = np.sum(np.abs(Jref), axis=1)
    with np.errstate(invalid="ignore"):
        bad = (Jref[:, 0] < 1e-7 * tot) | ((Jref[:, 1] > 0) & (Jref[:, 1] < 1e-7 * tot))
    return ~bad


def check_frequencies(F, Fref, tol=1e-6):
    nan_ref = ~np.isfinite(Fref)
    assert np.array_equal(~np.isfinite(F), nan_ref), "NaN pattern differs"
    ok = ~np.any(nan_ref, axis=1)
    F, Fref = F[ok], Fref[ok]
    scale = np.max(np.abs(Fref), axis=1, keepdims=True)
    err = np.abs(F - Fref)
    bound = tol * np.abs(Fref) + 1e-9 * scale
    worst = np.argmax(np.max(err / bound, axis=1))
    assert np.all(err <= bound), ("worst", F[worst], Fref[worst])
    return np.max(err / np.maximum(np.abs(Fref), 1e-300) * (np.abs(Fref) > 1e-6 * scale))


def check_angles(A, Aref, tol=1e-6):
    nan_ref = ~np.isfinite(Aref)
    assert np.array_equal(~np.isfinite(A), nan_ref), "NaN pattern differs"
    ok = ~np.any(nan_ref, axis=1)
    A, Aref = A[ok], Aref[ok]
    assert np.all((A >= 0) & (A < 2 * np.pi))
    d = np.abs(np.remainder(A - Aref + np.pi, 2 * np.pi) - np.pi)
    worst = np.argmax(np.max(d, axis=1))
    assert np.all(d <= tol), ("worst", A[worst], Aref[worst])
    return np.max(d)


@pytest.mark.parametrize("cfg", CFGS)
def test_angles_frequencies_fixed_focal_distance(cfg):
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "actions_%s.npz" % cfg))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, cfg + ".coef"))
    J, A, F = agama_b200.actions(pot, g["points"], fd=g["fd"], angles=True, frequencies=True)
    # the actions from the shared nodes are those of the actions-only path to round-off (the two
    # kernels inline the same potential evaluation, each with its own instruction schedule)
    J0 = agama_b200.actions(pot, g["points"], fd=g["fd"])
    assert np.array_equal(np.isfinite(J), np.isfinite(J0))
    fin = np.isfinite(J0)
    atol = 1e-14 * np.max(np.abs(J0[fin]))
    assert np.allclose(J[fin], J0[fin], rtol=1e-12, atol=atol), np.max(np.abs(J[fin] - J0[fin]))
    keep = well_conditioned(g["act_fd"])
    assert np.sum(~keep) <= 2
    print(cfg, "frequencies max rel %.2e" % check_frequencies(F[keep], g["freq_fd"][keep]),
          "angles max abs %.2e" % check_angles(A[keep], g["ang_fd"][keep]), "excluded", np.sum(~keep))


def test_angles_frequencies_through_the_finder_and_single_point():
    import ctypes
    import torch
    import agama_b200
    from agama_b200 import _native
    g = np.load(os.path.join(GOLDEN, "actions_cfg2.npz"))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg2.coef"))
    af = agama_b200.ActionFinder(pot)
    pts = g["points"]
    J, A, F = af(pts, angles=True, frequencies=True)
    _, fd = af(pts, fd=True)
    Js, As, Fs = agama_b200.actions(pot, pts, fd=fd, angles=True, frequencies=True)
    assert np.array_equal(J, Js, equal_nan=True) and np.array_equal(A, As, equal_nan=True)
    assert np.array_equal(F, Fs, equal_nan=True)
    # only angles / only frequencies, device buffers
    Ad = af(torch.tensor(pts, device="cuda"), actions=False, angles=True)
    Fd = af(torch.tensor(pts, device="cuda"), actions=False, frequencies=True)
    torch.cuda.synchronize()
    assert np.array_equal(Ad.cpu().numpy(), A, equal_nan=True) and np.array_equal(Fd.cpu().numpy(), F, equal_nan=True)
    # the reference-named single-point entry points
    p = np.ascontiguousarray(pts[7])
    act, ang, freq = np.zeros(3), np.zeros(3), np.zeros(3)
    _native.lib().agama_evalActionsAnglesFrequencies(af.handle, _native.ptr(p), _native.ptr(act), _native.ptr(ang),
                                                     _native.ptr(freq))
    assert np.array_equal(act, J[7]) and np.array_equal(ang, A[7]) and np.array_equal(freq, F[7])
    _native.lib().agama_evalActionsAnglesFrequenciesStandalone(pot.handle, ctypes.c_double(g["fd"][7]),
                                                              _native.ptr(p), None, _native.ptr(ang), None)
    assert np.allclose(ang, g["ang_fd"][7], rtol=0, atol=1e-6)
