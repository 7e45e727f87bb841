"""The C++ mirror of the reference's API (include/agama_b200.hpp, header-only over the C-ABI):
tests/cpp/cpp_api_check.cpp, compiled here with g++ against the engine's library, uses
potential::Multipole::eval, actions::ActionFinderAxisymFudge::actions (cylindrical input, as
the reference's finder) and orbit::integrate the way a reference C++ caller does.

CPU: the program compiles and links against the library with -Wall -Werror, and without a CUDA
device it reports the engine's error (there is no CPU fallback).  GPU: its potentials, actions,
orbits and trajectory against the reference's golden vectors and the Python API."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, GOLDEN, gpu_available

LIBDIR = os.path.join(ROOT, "agama_b200", "_lib")


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    if not os.path.exists(os.path.join(LIBDIR, "libagama_b200.so")):
        pytest.skip("engine library not built")
    exe = str(tmp_path_factory.mktemp("cpp") / "cpp_api_check")
    r = subprocess.run(["g++", "-std=c++11", "-O2", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "cpp_api_check.cpp"), "-o", exe, "-L" + LIBDIR,
                        "-lagama_b200", "-Wl,-rpath," + LIBDIR], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def run(program, tmp_path, pts3, pts6, coef="cfg2"):
    f3, f6, out = tmp_path / "p3.txt", tmp_path / "p6.txt", str(tmp_path / "out")
    np.savetxt(f3, pts3, fmt="%.17g")
    np.savetxt(f6, pts6, fmt="%.17g")
    r = subprocess.run([program, os.path.join(GOLDEN, coef + ".coef"), str(f3), str(f6), out],
                       capture_output=True, text=True, timeout=600)
    return r, out


@pytest.mark.skipif(gpu_available(), reason="checks the no-device behaviour")
def test_cpp_api_builds_and_refuses_without_device(program, tmp_path):
    r, _ = run(program, tmp_path, np.ones((2, 3)), np.ones((2, 6)))
    assert r.returncode == 3 and "CUDA" in r.stderr


@pytest.mark.gpu
def test_cpp_api_matches_reference_and_python_api(program, tmp_path):
    """potential and gradient at the golden points (1e-11: the points beyond r_max of config 2
    carry the outer asymptote's ~2e-12 conditioning, see test_potential_gpu), actions through the
    finder (1e-6 of the reference's finder), orbits and a trajectory equal to the Python API's
    (the same C-ABI calls) to round-off"""
    import agama_b200
    gp = np.load(os.path.join(GOLDEN, "potential_cfg2.npz"))
    ga = np.load(os.path.join(GOLDEN, "actions_cfg2.npz"))
    pts3, pts6 = gp["points"][:200], ga["points"][:200]
    r, out = run(program, tmp_path, pts3, pts6)
    assert r.returncode == 0, r.stderr
    pot = np.loadtxt(out + "_pot.txt").reshape(-1, 4)
    act = np.loadtxt(out + "_act.txt").reshape(-1, 3)
    orb = np.loadtxt(out + "_orb.txt").reshape(-1, 6)
    traj = np.loadtxt(out + "_traj.txt").reshape(-1, 7)
    assert np.all(np.abs(pot[:, 0] - gp["phi"][:200]) <= 1e-11 * np.abs(gp["phi"][:200]))
    gerr = np.linalg.norm(pot[:, 1:] - gp["grad"][:200], axis=1) / np.linalg.norm(gp["grad"][:200], axis=1)
    assert gerr.max() <= 1e-11, gerr.max()
    Jref = ga["act_finder"][:200]
    assert np.array_equal(np.isfinite(act), np.isfinite(Jref))
    ok = np.all(np.isfinite(Jref), axis=1)
    scale = np.sum(np.abs(Jref[ok]), axis=1, keepdims=True)
    assert np.all(np.abs(act[ok] - Jref[ok]) <= 1e-6 * np.abs(Jref[ok]) + 1e-9 * scale)
    p = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg2.coef"))
    fin = agama_b200.orbit(p, pts6, np.ones(len(pts6)))
    good = np.all(np.isfinite(fin), axis=1)
    assert np.array_equal(good, np.all(np.isfinite(orb), axis=1))
    assert np.allclose(orb[good], fin[good], rtol=1e-10, atol=1e-10 * np.abs(fin[good]).max())
    times, tr = agama_b200.trajectory(p, pts6[:1], 1.0, 11)
    assert traj.shape == (11, 7)
    assert np.allclose(traj[:, 0], times[0], rtol=1e-15, atol=1e-15)
    assert np.allclose(traj[:, 1:], tr[0], rtol=1e-10, atol=1e-10 * np.abs(tr[0]).max())
