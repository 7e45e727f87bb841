"""Parity of the device Staeckel-fudge actions with the reference (golden vectors from
tests/golden/make_golden.py: actions::evalAxisymFudge for given focal distances, and
ActionFinderAxisymFudge with its own focal-distance table).

Bound (engine specification): actions agree to 1e-6 relative.  For components that vanish
(Jr of a circular orbit, Jz of a planar one) the bound is taken relative to the total action
|Jr| + |Jz| + |Jphi|: |dJ_i| <= 1e-6 |J_i| + 1e-9 (|Jr| + |Jz| + |Jphi|).
Unbound points (E >= 0) give NaN for Jr, Jz in both."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CFGS = ["cfg2", "cfg5", "cfg4"]


def check_actions(J, Jref, tol=1e-6):
    nan_ref = ~np.isfinite(Jref)
    assert np.array_equal(~np.isfinite(J), nan_ref), "NaN pattern differs"
    ok = ~np.any(nan_ref, axis=1)
    J, Jref = J[ok], Jref[ok]
    scale = np.sum(np.abs(Jref), axis=1, keepdims=True)
    err = np.abs(J - Jref)
    bound = tol * np.abs(Jref) + 1e-9 * scale
    worst = np.argmax(np.max(err / bound, axis=1))
    assert np.all(err <= bound), ("worst", J[worst], Jref[worst], np.max(err / bound))
    return np.max(err / np.maximum(np.abs(Jref), 1e-300) * (np.abs(Jref) > 1e-6 * scale))


def tables(g):
    return {k[4:]: g[k] for k in g.files if k.startswith("tab_")}


@pytest.mark.parametrize("cfg", CFGS)
def test_actions_fixed_focal_distance(cfg):
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "actions_%s.npz" % cfg))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, cfg + ".coef"))
    J = agama_b200.actions(pot, g["points"], fd=g["fd"])
    check_actions(J, g["act_fd"])


@pytest.mark.parametrize("cfg", CFGS)
def test_action_finder(cfg):
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "actions_%s.npz" % cfg))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, cfg + ".coef"))
    af = agama_b200.ActionFinder(pot, tables=tables(g))
    J, fd = af(g["points"], fd=True)
    # the focal distance comes from the same bilinear table: round-off level agreement (where
    # the table is ~0 the sign of the round-off decides between a tiny Delta and max(0, .) = 0)
    fin = np.isfinite(g["fd"])
    assert np.allclose(fd[fin], g["fd"][fin], rtol=1e-10, atol=1e-8 * np.max(g["fd"][fin]))
    check_actions(J, g["act_finder"])


@pytest.mark.parametrize("cfg", CFGS)
def test_action_finder_builds_own_tables(cfg):
    """agama_createActionFinder: the engine builds the focal-distance table from shell orbits on
    the device and the L_circ(E) interpolator itself; the grids must equal the reference's, the
    focal distances agree to the shell-orbit root tolerance, and the actions to 1e-6."""
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "actions_%s.npz" % cfg))
    ref_tab = tables(g)
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, cfg + ".coef"))
    af = agama_b200.ActionFinder(pot)
    tab = af.tables()
    J = af(g["points"])
    report = {}
    report["gridE"] = np.max(np.abs(tab["gridE"] / ref_tab["gridE"] - 1))
    for k in ("lofe", "rofl", "phiofr"):
        report[k] = np.max(np.abs(tab[k][:3] - ref_tab[k][:3]) / np.maximum(np.abs(ref_tab[k][:3]), 1e-300))
    # Delta per node over the energy rows that the test points use (one row of margin each side),
    # relative to the row's typical value.  Rows far outside (E -> 0: shell orbits at r ~ 1e10 and
    # beyond) hold meaningless values up to 1e36 in both tables.  Within the rows used the nodes
    # agree to ~5e-7 (the shell radius is a root located to 1e-6 of its bracket; near circular
    # orbits the focal-distance formula divides two vanishing quantities).
    pts = g["points"]
    E = pot.potential(pts[:, :3]) + 0.5 * np.sum(pts[:, 3:] ** 2, axis=1)
    xi = np.log(ref_tab["invPhi0"] - 1 / E[E < 0])
    r0 = max(0, np.searchsorted(ref_tab["gridE"], np.min(xi)) - 2)
    r1 = min(len(ref_tab["gridE"]), np.searchsorted(ref_tab["gridE"], np.max(xi)) + 1)
    dref, dnew = ref_tab["delta"][r0:r1], tab["delta"][r0:r1]
    typical = np.array([np.median(row[row > 0]) if np.any(row > 0) else 1.0 for row in dref])[:, None]
    rel = np.abs(dnew - dref) / np.maximum(dref, typical)
    report["rows"] = (r0, r1)
    report["delta"] = np.max(rel)
    report["delta_node"] = np.unravel_index(np.argmax(rel), rel.shape)
    print(cfg, report)
    check_actions(J, g["act_finder"])
    assert tab["gridE"].shape == ref_tab["gridE"].shape and tab["lofe"].shape == ref_tab["lofe"].shape
    # grids to round-off (the L_circ grid of config 2 ends in the NFW outer asymptote whose
    # condition number ~1e4 moves a few single-precision grid steps by one float ulp: 1e-8)
    assert report["gridE"] <= 1e-12 and report["lofe"] <= 1e-7
    assert report["delta"] <= 1e-5


def test_actions_device_pointers_and_single_point():
    import ctypes
    import torch
    import agama_b200
    from agama_b200 import _native
    g = np.load(os.path.join(GOLDEN, "actions_cfg2.npz"))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg2.coef"))
    af = agama_b200.ActionFinder(pot, tables=tables(g))
    host = af(g["points"])
    dev = af(torch.tensor(g["points"], device="cuda"))
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy(), host, equal_nan=True)
    # the reference-named single-point entry points
    p = np.ascontiguousarray(g["points"][5])
    act = np.zeros(3)
    _native.lib().agama_evalActionsAnglesFrequencies(af.handle, _native.ptr(p), _native.ptr(act), None, None)
    assert np.array_equal(act, host[5])
    _native.lib().agama_evalActionsAnglesFrequenciesStandalone(pot.handle, ctypes.c_double(g["fd"][5]),
                                                              _native.ptr(p), _native.ptr(act), None, None)
    assert np.allclose(act, g["act_fd"][5], rtol=1e-6)


def test_actions_reject_non_axisymmetric():
    import agama_b200
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg1.coef"))
    with pytest.raises(RuntimeError, match="axisymmetric"):
        agama_b200.actions(pot, np.ones((2, 6)), fd=1.0)


@pytest.mark.parametrize("cfg", CFGS)
def test_action_finder_mixed_precision(cfg):
    """FP32 integrand arithmetic and compensated FP32 Gauss-Legendre sums (F(tau), the potential
    and the roots in FP64): within the 1e-6 bound of the reference, and within 1e-6 of the FP64
    form (measured on B200: a few 1e-7 at most, reported here per configuration)"""
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "actions_%s.npz" % cfg))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, cfg + ".coef"))
    af = agama_b200.ActionFinder(pot, tables=tables(g))
    J64 = af(g["points"])
    agama_b200.set_action_precision(True)
    try:
        J32 = af(g["points"])
    finally:
        agama_b200.set_action_precision(False)
    assert not np.array_equal(J32, J64, equal_nan=True)          # the mixed path did run
    check_actions(J32, g["act_finder"])
    err = check_actions(J32, J64)
    print(cfg, "mixed-precision actions vs FP64: max relative error %.3g" % err)
    assert np.array_equal(af(g["points"]), J64, equal_nan=True)  # the setting is off again


@pytest.mark.parametrize("cfg", ["cfg4", "cfg5"])
def test_mixed_precision_loosely_bound_orbits(cfg):
    """the mixed-precision integrand on orbits reaching far out (apocentres up to ~1e6, where
    (tau - Delta^2)^2 tau exceeds the FP32 range): within 1e-6 of the FP64 form"""
    import agama_b200
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, cfg + ".coef"))
    af = agama_b200.ActionFinder(pot)
    rng = np.random.default_rng(17)
    R = 10 ** rng.uniform(-1, 4, 400)
    pos = np.column_stack([R, np.zeros_like(R), 0.3 * R * rng.uniform(-1, 1, 400)])
    vesc = np.sqrt(-2 * pot.potential(pos))
    u = rng.uniform(0.3, 0.995, 400)
    d = rng.normal(size=(400, 3))
    vel = d / np.linalg.norm(d, axis=1)[:, None] * (u * vesc)[:, None]
    pts = np.hstack([pos, vel])
    J64 = af(pts)
    agama_b200.set_action_precision(True)
    try:
        J32 = af(pts)
    finally:
        agama_b200.set_action_precision(False)
    err = check_actions(J32, J64)
    print(cfg, "loosely bound orbits, mixed vs FP64: %.3g" % err)
