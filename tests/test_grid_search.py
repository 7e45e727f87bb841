"""The device form of the grid search (binSearchScaled in agama_b200/csrc/common.cuh: a multiplied
first guess, a short walk to the neighbouring segment, then the bisection) built for the host
(tests/cpp/grid_search_check.cpp) returns the segment of binSearch, the restatement of the
reference's math::binSearch (src/math_core.cpp:251-280), for every node, its floating-point
neighbours, random points over and beyond the grid, NaN and the infinities, on uniform,
geometric, irregular and the Multipole tau grids (CPU, no GPU)."""
import os
import subprocess
import tempfile

from conftest import ROOT


def test_scaled_search_equals_bisection():
    exe = os.path.join(tempfile.mkdtemp(), "grid_search_check")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-Wno-unknown-pragmas", "-x", "c++",
                        "-I" + os.path.join(ROOT, "agama_b200", "csrc"),
                        os.path.join(ROOT, "tests", "cpp", "grid_search_check.cpp"), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "mismatches 0" in out.stdout, out.stdout
