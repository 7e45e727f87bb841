"""Parity of the density and radius entry points with the reference's plain-C interface
(agama_evalDensity, agama_R_circ, agama_R_from_Lz, agama_R_max, agama_findPlanarOrbitExtent;
golden vectors from the reference through that same interface, tests/golden/make_golden.py).

Potentials: config 1 (triaxial: the radius routines average it over 17 azimuths, 9 with the
y-reflection mirror), config 2 (axisymmetric), quad (lmax = 2, 1-D splines), sph (spherical) and
lop (no symmetry, off-centre: energies below the minimum of the averaged potential give NaN).

Tolerances: radii 1e-8 relative (the reference's root finders stop at 1e-10 in a scaled variable
whose derivative dR/R ds is at most ~10 there, and a one-ulp difference in a bracket value may send
the search one iteration another way), with NaN and infinity where the reference has them.
Density 1e-9 relative where |rho| is not dominated by cancellation (the Laplacian is a sum of
second derivatives known to 1e-9 relative of the Hessian), and 0 exactly where the reference's
round-off test returns 0."""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

NAMES = ["cfg1", "cfg2", "quad", "sph", "lop"]


def same_nonfinite(a, b):
    return np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(np.isposinf(a), np.isposinf(b))


def rel(a, b):
    ok = np.isfinite(b)
    return np.abs(a[ok] - b[ok]) / np.maximum(np.abs(b[ok]), 1e-300)


@pytest.fixture(scope="module", params=NAMES)
def case(request):
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "utils_%s.npz" % request.param))
    return request.param, agama_b200.Potential(file=os.path.join(GOLDEN, request.param + ".coef")), g


def test_density(case):
    name, pot, g = case
    rho = pot.density(g["points"])
    ref = g["rho"]
    assert same_nonfinite(rho, ref), name
    assert np.array_equal(rho == 0, ref == 0), name
    err = rel(rho, ref)
    big = np.abs(ref[np.isfinite(ref)]) > 1e-6 * np.median(np.abs(ref[np.isfinite(ref)]))
    assert np.max(err[big]) <= 1e-9, (name, np.max(err[big]))
    assert np.max(err) <= 1e-6, (name, np.max(err))


def test_rcirc_rmax(case):
    name, pot, g = case
    for got, ref in ((pot.Rcirc(E=g["E"]), g["Rcirc"]), (pot.Rmax(g["E"]), g["Rmax"]),
                     (pot.Rcirc(L=g["L"]), g["RfromLz"])):
        assert same_nonfinite(got, ref), name
        assert np.max(rel(got, ref)) <= 1e-8, (name, np.max(rel(got, ref)))


def test_periapo(case):
    name, pot, g = case
    got = pot.Rperiapo(g["EL"])
    ref = g["periapo"]
    assert same_nonfinite(got, ref), name
    assert np.max(rel(got, ref)) <= 1e-8, (name, np.max(rel(got, ref)))


def test_scalar_c_entry_points():
    """the reference-named scalar calls against the batched ones, on config 1"""
    import agama_b200
    from agama_b200 import _native
    g = np.load(os.path.join(GOLDEN, "utils_cfg1.npz"))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg1.coef"))
    L = _native.lib()
    for k in (3, 40, 77):
        assert L.agama_R_circ(pot.handle, g["E"][k]) == pytest.approx(g["Rcirc"][k], rel=1e-8)
        assert L.agama_R_max(pot.handle, g["E"][k]) == pytest.approx(g["Rmax"][k], rel=1e-8)
        assert L.agama_R_from_Lz(pot.handle, g["L"][k]) == pytest.approx(g["RfromLz"][k], rel=1e-8)
        r1, r2 = ctypes.c_double(), ctypes.c_double()
        L.agama_findPlanarOrbitExtent(pot.handle, g["EL"][k, 0], g["EL"][k, 1], ctypes.byref(r1), ctypes.byref(r2))
        assert (r1.value, r2.value) == pytest.approx(tuple(g["periapo"][k]), rel=1e-8)
        p = np.ascontiguousarray(g["points"][k])
        rho = L.agama_evalDensity(pot.handle, p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0.0)
        assert rho == pytest.approx(g["rho"][k], rel=1e-9)


def test_device_variants():
    import torch
    import agama_b200
    from agama_b200 import _native, _dev_ptr, _current_stream
    g = np.load(os.path.join(GOLDEN, "utils_cfg2.npz"))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg2.coef"))
    rho = pot.density(torch.tensor(g["points"], device="cuda"))
    assert np.array_equal(rho.cpu().numpy(), pot.density(g["points"]))
    EL = torch.tensor(g["EL"], device="cuda")
    E, Lz = EL[:, 0].contiguous(), EL[:, 1].contiguous()
    r1, r2 = torch.empty_like(E), torch.empty_like(E)
    rc = _native.lib().agama_potentialRadiiManyDevice(pot.handle, 3, len(E), _dev_ptr(E), _dev_ptr(Lz),
                                                      _dev_ptr(r1), _dev_ptr(r2), _current_stream())
    assert rc == 0, _native.error()
    got = torch.stack([r1, r2], dim=1).cpu().numpy()
    assert np.array_equal(np.nan_to_num(got, nan=-1), np.nan_to_num(pot.Rperiapo(g["EL"]), nan=-1))
    rc = _native.lib().agama_potentialRadiiManyDevice(pot.handle, 7, 1, _dev_ptr(E), None, _dev_ptr(r1), None,
                                                      _current_stream())
    assert rc != 0 and "unknown query" in _native.error()
