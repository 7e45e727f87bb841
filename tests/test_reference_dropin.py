"""The engine behind the reference's own C++ interfaces (include/agama_b200_reference.hpp):
tests/cpp/reference_dropin_check.cpp, built by oracle/Makefile against the reference's headers and
objects (without the reference's plain-C interface) and the engine's library, holds a
potential::PtrPotential to the engine's MultipoleB200 beside one to the reference's own Multipole
read from the same coefficient file, and an actions::PtrActionFinder to the engine's finder.

CPU: without a CUDA device the program reports the engine's error (no CPU fallback).
GPU: through the reference's eval front-ends (Cartesian, cylindrical, spherical) the engine's
potential, gradient and Hessian equal the reference's (1e-11 relative for the value and the
gradient: the points beyond r_max of config 2 carry the outer asymptote's ~2e-12 conditioning;
Hessian 1e-9 of its norm); the reference's R_circ and standalone fudge on the engine's potential
equal those on its own (1e-10); the batched density override equals the reference's loop (1e-9);
the engine's finder through BaseActionFinder matches the reference's golden actions (1e-6)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, GOLDEN, gpu_available

PROGRAM = os.path.join(ROOT, "oracle", "_ref", "reference_dropin_check")
needs_program = pytest.mark.skipif(not os.path.exists(PROGRAM),
                                   reason="oracle/_ref/reference_dropin_check not built (needs the reference sources)")


def run(tmp_path, n3=200, n6=200):
    gp = np.load(os.path.join(GOLDEN, "potential_cfg2.npz"))
    ga = np.load(os.path.join(GOLDEN, "actions_cfg2.npz"))
    f3, f6, ffd = tmp_path / "p3.txt", tmp_path / "p6.txt", tmp_path / "fd.txt"
    np.savetxt(f3, gp["points"][:n3], fmt="%.17g")
    np.savetxt(f6, ga["points"][:n6], fmt="%.17g")
    np.savetxt(ffd, ga["fd"][:n6], fmt="%.17g")
    out = str(tmp_path / "out")
    r = subprocess.run([PROGRAM, os.path.join(GOLDEN, "cfg2.coef"), str(f3), str(f6), str(ffd), out],
                       capture_output=True, text=True, timeout=900)
    return r, out, gp, ga


@needs_program
@pytest.mark.skipif(gpu_available(), reason="checks the no-device behaviour")
def test_reference_dropin_refuses_without_device(tmp_path):
    r, _, _, _ = run(tmp_path, 2, 2)
    assert r.returncode == 3 and "CUDA" in r.stderr, (r.returncode, r.stderr)


def _rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


@needs_program
@pytest.mark.gpu
def test_reference_dropin_matches_reference(tmp_path):
    r, out, gp, ga = run(tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "potentials: Multipole (engine) / Multipole (reference)" in r.stdout
    pot = np.loadtxt(out + "_pot.txt")
    assert _rel(pot[:, 0], pot[:, 4]).max() <= 1e-11      # 2e-12 beyond r_max of config 2 (outer power law)
    gerr = np.linalg.norm(pot[:, 1:4] - pot[:, 5:8], axis=1) / np.linalg.norm(pot[:, 5:8], axis=1)
    assert gerr.max() <= 1e-11, gerr.max()
    assert _rel(pot[:, 4], gp["phi"][:len(pot)]).max() == 0          # the reference side is the golden one
    hess = np.loadtxt(out + "_hess.txt")
    herr = np.linalg.norm(hess[:, :6] - hess[:, 6:], axis=1) / np.linalg.norm(hess[:, 6:], axis=1)
    assert herr.max() <= 1e-9, herr.max()
    cyl = np.loadtxt(out + "_cyl.txt")
    assert _rel(cyl[:, 0], cyl[:, 10]).max() <= 1e-11
    gcyl = np.linalg.norm(cyl[:, 1:4] - cyl[:, 11:14], axis=1) / np.linalg.norm(cyl[:, 11:14], axis=1)
    hcyl = np.linalg.norm(cyl[:, 4:10] - cyl[:, 14:20], axis=1) / np.linalg.norm(cyl[:, 14:20], axis=1)
    assert gcyl.max() <= 1e-11 and hcyl.max() <= 1e-9, (gcyl.max(), hcyl.max())
    sph = np.loadtxt(out + "_sph.txt")
    gsph = np.linalg.norm(sph[:, 1:4] - sph[:, 5:8], axis=1) / np.linalg.norm(sph[:, 5:8], axis=1)
    assert _rel(sph[:, 0], sph[:, 4]).max() <= 1e-11 and gsph.max() <= 1e-11, gsph.max()
    rc = np.loadtxt(out + "_rc.txt")
    assert _rel(rc[:, 1], rc[:, 2]).max() <= 1e-10
    fud = np.loadtxt(out + "_fud.txt")
    ok = np.isfinite(fud[:, 3:]).all(1)
    assert np.array_equal(np.isfinite(fud[:, :3]), np.isfinite(fud[:, 3:]))
    scale = np.abs(fud[ok, 3:]).sum(1, keepdims=True)
    assert np.all(np.abs(fud[ok, :3] - fud[ok, 3:]) <= 1e-10 * scale)
    rho = np.loadtxt(out + "_rho.txt")
    good = np.isfinite(rho[:, 1]) & (rho[:, 1] != 0)
    assert np.abs(rho[good, 0] - rho[good, 1]).max() <= 1e-9 * np.abs(rho[good, 1]).max()
    act = np.loadtxt(out + "_act.txt")
    assert np.array_equal(act[:, :3], act[:, 3:], equal_nan=True)     # one point and a batch agree
    Jref = ga["act_finder"][:len(act)]
    assert np.array_equal(np.isfinite(act[:, :3]), np.isfinite(Jref))
    ok = np.isfinite(Jref).all(1)
    scale = np.abs(Jref[ok]).sum(1, keepdims=True)
    assert np.all(np.abs(act[ok, :3] - Jref[ok]) <= 1e-6 * np.abs(Jref[ok]) + 1e-9 * scale)
