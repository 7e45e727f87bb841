"""CPU tests of the C-ABI library: it loads, exports every symbol declared in
include/agama_b200.h, parses coefficient files on the host, and refuses to compute without a
CUDA device (there is no CPU fallback)."""
import ctypes
import os
import re

import pytest

from agama_b200 import _native
from conftest import ROOT, GOLDEN, gpu_available


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "agama_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(agama_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = _native.lib()
    names = declared_symbols()
    assert len(names) >= 8
    for name in names:
        assert hasattr(lib, name), name
    # the Python loader declares argument types for every exported entry point
    assert set(names) <= set(_native.SIGNATURES)


@pytest.mark.parametrize("name,lmax,mmax,sym,nt", [
    ("cfg1", 6, 6, 15, 25), ("cfg2", 8, 0, 31, 31), ("cfg3", 8, 8, 15, 31), ("cfg5", 12, 0, 31, 43),
    ("quad", 2, 2, 15, 0), ("sph", 0, 0, 63, 0)])
def test_coefficient_file_host_parse(name, lmax, mmax, sym, nt):
    v = [ctypes.c_int() for _ in range(5)]
    rc = _native.lib().agama_inspectMultipoleFile(os.path.join(GOLDEN, name + ".coef").encode(),
                                                  *[ctypes.byref(x) for x in v])
    assert rc == 0, _native.error()
    assert [x.value for x in v][:3] == [lmax, mmax, sym]
    assert v[4].value == nt            # tau grid: 3 (lmax+2) + 1 nodes for the 2-D splines


def test_bad_file_reports_error():
    rc = _native.lib().agama_inspectMultipoleFile(b"/nonexistent.coef", None, None, None, None, None)
    assert rc != 0 and "cannot open" in _native.error()


def test_unsupported_parameters_rejected():
    h = _native.lib().agama_createPotential(b"type=Plummer, mass=1")
    assert not h
    assert "Multipole" in _native.error() or "not supported" in _native.error()


def test_density_objects_not_constructed():
    """density models only construct potentials, which come from coefficient files here"""
    L = _native.lib()
    assert not L.agama_createDensity(b"type=Plummer, mass=1")
    assert "agama_evalDensity" in _native.error()
    L.agama_deleteDensity(None)


@pytest.mark.skipif(gpu_available(), reason="checks the no-device behaviour")
def test_no_cpu_fallback():
    h = _native.lib().agama_createPotential(("file=" + os.path.join(GOLDEN, "cfg1.coef")).encode())
    assert not h
    assert "CUDA" in _native.error()
