"""The engine's restated numerics against the reference's own routines (CPU, no GPU).

Built for the host with the reference's flags (tests/cpp/numerics_check.cpp), the engine's
normalised Legendre functions with their first and second derivatives (sphharm.cuh, restating
math::sphHarmArray, src/math_sphharm.cpp:63-132, including its small-sin(theta) branches), the
multiple-angle recurrence (math::trigMultiAngle, :134-154; its first sine and cosine come from the C
library here, from the reference's own sincos there) and the interval scalings (math::unscale /
scale for the doubly infinite, semi-infinite and cubic-stretch maps, src/math_core.cpp:296-396) must
give the reference's values, called through the oracle library, to round-off."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

ref = pytest.importorskip("oracle.ref")
pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
D = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def run():
    import tempfile
    exe = os.path.join(tempfile.mkdtemp(), "numerics_check")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-march=x86-64-v3", "-Wall", "-Werror", "-Wno-unknown-pragmas",
                        "-x", "c++", "-I" + os.path.join(ROOT, "agama_b200", "csrc"),
                        os.path.join(ROOT, "tests", "cpp", "numerics_check.cpp"), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

    def go(lines):
        out = subprocess.run([exe], input="\n".join(lines) + "\n", capture_output=True, text=True, timeout=60)
        assert out.returncode == 0, out.stderr
        return [np.array([float(v) for v in line.split()]) for line in out.stdout.splitlines()]
    return go


def close(a, b, rel=4e-15):
    """equal, or within rel of b (infinities must be equal)"""
    with np.errstate(invalid="ignore"):
        return np.all((a == b) | (np.abs(a - b) <= rel * np.maximum(np.abs(b), 1e-300)))


def test_legendre_functions(run):
    L = ref.lib()
    L.ref_sph_harm_array.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, D, D, D]
    rng = np.random.default_rng(3)
    taus = np.concatenate([rng.uniform(-1, 1, 40), [0.0, 1e-9, -1e-9, 1 - 1e-9, -1 + 1e-9, 1 - 1e-17, 0.9999999,
                                                   -0.9999999, 1.0, -1.0]])
    cases = [(lmax, m, t) for lmax in (0, 1, 2, 6, 8, 12, 16) for m in sorted({0, 1, 2, lmax // 2, lmax}) if m <= lmax
             for t in taus]
    got = run(["L %d %d %.17g" % c for c in cases])
    exact = 0
    for (lmax, m, t), g in zip(cases, got):
        n = lmax - m + 1
        P, dP, d2P = np.zeros(n), np.zeros(n), np.zeros(n)
        assert L.ref_sph_harm_array(lmax, m, t, P.ctypes.data_as(D), dP.ctypes.data_as(D), d2P.ctypes.data_as(D)) == 0
        want = np.column_stack([P, dP, d2P]).ravel()
        # round-off relative to the largest of the array's values and derivatives
        sc = np.abs(want).max() + 1e-300
        assert np.all(np.abs(g - want) <= 1e-13 * sc), (lmax, m, t, np.abs(g - want).max() / sc)
        exact += np.array_equal(g, want)
    assert exact >= 0.5 * len(cases), (exact, len(cases))


def test_multiple_angles(run):
    L = ref.lib()
    L.ref_trig_multi_angle.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, D]
    rng = np.random.default_rng(4)
    cases = [(phi, m, ns) for phi in np.concatenate([rng.uniform(-7, 7, 30), [0.0, np.pi, -np.pi / 2, 1e-12]])
             for m in (1, 2, 6, 12, 16) for ns in (0, 1)]
    got = run(["T %.17g %d %d" % c for c in cases])
    for (phi, m, ns), g in zip(cases, got):
        out = np.zeros(2 * m if ns else m)
        L.ref_trig_multi_angle(phi, m, ns, out.ctypes.data_as(D))
        # the recurrence starts from sin / cos of phi and phi / 2: the reference's own sincos
        # (src/math_core.cpp:171-207) against the C library's, an ulp apart at most
        assert np.all(np.abs(g - out) <= 1e-14), (phi, m, ns, np.abs(g - out).max())


def test_scalings(run):
    L = ref.lib()
    L.ref_unscale.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, D, D]
    L.ref_scale.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, D]
    rng = np.random.default_rng(5)
    s = np.concatenate([rng.uniform(0, 1, 60), [1e-6, 0.5, 1 - 1e-6]])
    cases = [(k, a, b, x) for k, a, b in ((0, 0.0, 0.0), (1, 2.5, 0.0), (1, 1e-3, 0.0), (2, 0.3, 7.0), (2, -2.0, 1e3))
             for x in s]
    got = run(["U %d %.17g %.17g %.17g" % c for c in cases])
    u, du = ctypes.c_double(), ctypes.c_double()
    for (k, a, b, x), g in zip(cases, got):
        L.ref_unscale(k, a, b, x, ctypes.byref(u), ctypes.byref(du))
        assert close(g, np.array([u.value, du.value])), (k, a, b, x, g, u.value, du.value)
    ucases = [(0.3, 7.0, x) for x in rng.uniform(0.3, 7.0, 60)] + [(-2.0, 1e3, x) for x in rng.uniform(-2, 1e3, 60)] + \
        [(0.3, 7.0, 0.3), (0.3, 7.0, 7.0), (0.3, 7.0, 3.65)]
    got = run(["S %.17g %.17g %.17g" % c for c in ucases])
    sv = ctypes.c_double()
    for (a, b, x), g in zip(ucases, got):
        L.ref_scale(2, a, b, x, ctypes.byref(sv))
        # the engine inverts the cubic stretch by Newton steps from its own first guess: the same
        # s to round-off of the map (ds ~ eps / (du/ds))
        assert abs(g[0] - sv.value) <= 1e-12, (a, b, x, g[0], sv.value)
