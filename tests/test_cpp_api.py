"""The C++ mirror of the reference's API (include/agama_b200.hpp, header-only over the C-ABI):
tests/cpp/cpp_api_check.cpp, compiled here with g++ against the engine's library, uses
potential::Multipole::eval, actions::ActionFinderAxisymFudge::actions (cylindrical input, as
the reference's finder) and orbit::integrate the way a reference C++ caller does.

Here (CPU): the program compiles and links against the library with -Wall -Werror, and without a
CUDA device it reports the engine's error (there is no CPU fallback).  The numbers behind the
header are those of the C-ABI entry points that the GPU tests check."""
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
