"""The coefficient-file writer (agama_writePotential / agama_writeMultipoleCoefs / Potential.export):
the reference's writePotentialMultipole layout (src/potential_factory.cpp:909-930) with numbers in
17 significant digits.

CPU: coefficients parsed from the reference's own files are written back host-only; the engine's
host parser reads the same order, symmetry and grids from them, and the reference built here
(oracle) reads them into a potential that evaluates bit for bit as the one from the original file
(the written numbers round-trip to the same doubles).
GPU: Potential(file).export() then Potential(exported) evaluates bit for bit as the original."""
import ctypes
import os

import numpy as np
import pytest

from agama_b200 import _native
from conftest import GOLDEN

NAMES = ["cfg1", "cfg2", "cfg5", "quad", "sph", "lop"]


def parse_coef(path):
    """radii, Phi, dPhi (numCoefs x gridSizeR, index l(l+1)+m) of a Multipole coefficient file"""
    lines = [l.strip() for l in open(path)]
    n = int(next(l for l in lines if l.lower().startswith("gridsizer=")).split("=")[1])

    def block(tag):
        k = lines.index(tag) + 1
        head = lines[k].split("\t")[1:]
        idx = [int(h.split(",")[0][2:]) * (int(h.split(",")[0][2:]) + 1) + int(h.split(",")[1][2:]) for h in head]
        rows = np.array([[float(x) for x in lines[k + 1 + i].split("\t")] for i in range(n)])
        lmax = int(np.ceil(np.sqrt(max(idx) + 1))) - 1
        C = np.zeros(((lmax + 1) ** 2, n))
        for j, c in enumerate(idx):
            C[c] = rows[:, j + 1]
        return rows[:, 0], C
    r, P = block("#Phi")
    _, D = block("#dPhi/dr")
    return r, P, D


def write_host(path, r, P, D):
    P, D = np.ascontiguousarray(P), np.ascontiguousarray(D)
    rc = _native.lib().agama_writeMultipoleCoefs(str(path).encode(), len(r), _native.ptr(np.ascontiguousarray(r)),
                                                  P.shape[0], _native.ptr(P), _native.ptr(D))
    assert rc == 0, _native.error()


def inspect(path):
    v = [ctypes.c_int() for _ in range(5)]
    assert _native.lib().agama_inspectMultipoleFile(str(path).encode(), *[ctypes.byref(x) for x in v]) == 0, \
        _native.error()
    return [x.value for x in v]


@pytest.mark.parametrize("name", NAMES)
def test_written_file_round_trips_on_host(name, tmp_path):
    src = os.path.join(GOLDEN, name + ".coef")
    r, P, D = parse_coef(src)
    out = tmp_path / (name + ".coef")
    write_host(out, r, P, D)
    assert inspect(out) == inspect(src)
    r2, P2, D2 = parse_coef(out)
    assert np.array_equal(r2, r) and np.array_equal(P2, P) and np.array_equal(D2, D)
    ref = pytest.importorskip("oracle.ref")
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    pts = np.load(os.path.join(GOLDEN, "potential_%s.npz" % name))["points"][::9]
    a = ref.Potential(file=src).eval(pts, hess=True, nthreads=1)
    b = ref.Potential(file=str(out)).eval(pts, hess=True, nthreads=1)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_writer_rejects_bad_input(tmp_path):
    r = np.array([1.0, 2.0, 3.0])
    P = np.zeros((3, 3))          # 3 coefficients: not (lmax+1)^2
    rc = _native.lib().agama_writeMultipoleCoefs(str(tmp_path / "x.coef").encode(), 3, _native.ptr(r), 3,
                                                  _native.ptr(P), _native.ptr(P))
    assert rc != 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cfg1", "cfg2", "lop"])
def test_export_from_device_potential(name, tmp_path):
    import agama_b200
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, name + ".coef"))
    out = tmp_path / "exported.coef"
    pot.export(out)
    again = agama_b200.Potential(file=str(out))
    pts = np.load(os.path.join(GOLDEN, "potential_%s.npz" % name))["points"]
    a = pot.eval(pts, pot=True, acc=True, der=True)
    b = again.eval(pts, pot=True, acc=True, der=True)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
