"""ctypes wrapper over oracle/_ref/libagama_ref.so -- the reference Agama library compiled
from its own sources (see oracle/Makefile) plus the flat C driver in oracle/ref_driver.cpp.

TEST INFRASTRUCTURE ONLY.  Importable from tests/, from the golden-fixture generator and
from the CPU reference arm of bench.py; the B200 engine (agama_b200/) never imports it.

Every function below forwards to the reference's own code path for the hot path:
  eval_many            BasePotential::eval(PosCar)            potential_base.h:153-156
  orbits_many          orbit::OrbitIntegrator<Car>::run       orbit.cpp:52-84 (DOP853, math_ode.cpp:107-406)
  actions_fd_many      actions::evalAxisymFudge               actions_staeckel.cpp:683-693
  ActionFinder.actions actions::ActionFinderAxisymFudge::eval actions_staeckel.cpp:954-979
  CInterfacePotential  the reference's plain-C interface       interface_c.cpp:31-111
                       (density, R_circ, R_from_Lz, R_max, findPlanarOrbitExtent)
  ref_find_root_poly   math::findRoot on a polynomial          math_core.cpp:895-1041
  ref_sph_harm_array   math::sphHarmArray                      math_sphharm.cpp:63-132
  ref_trig_multi_angle math::trigMultiAngle                    math_sphharm.cpp:134-154
  ref_unscale / _scale math::unscale / scale                   math_core.cpp:296-396
                       (called through lib() by tests/test_rootsearch.py, test_numerics_oracle.py)
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "_ref", "libagama_ref.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_L = ctypes.POINTER(ctypes.c_long)
_LL = ctypes.POINTER(ctypes.c_longlong)
_I = ctypes.POINTER(ctypes.c_int)


def available():
    return os.path.exists(LIBPATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle library not built: run `make -C oracle` (needs the reference sources)")
        L = ctypes.CDLL(LIBPATH)
        L.ref_error.restype = ctypes.c_char_p
        L.ref_load_potential.restype = ctypes.c_void_p
        L.ref_load_potential.argtypes = [ctypes.c_char_p]
        L.ref_create_potential.restype = ctypes.c_void_p
        L.ref_create_potential.argtypes = [ctypes.c_char_p]
        L.ref_write_potential.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.ref_free_potential.argtypes = [ctypes.c_void_p]
        L.ref_eval_many.argtypes = [ctypes.c_void_p, ctypes.c_long, _D, _D, _D, _D, ctypes.c_int]
        L.ref_eval_cyl_many.argtypes = [ctypes.c_void_p, ctypes.c_long, _D, _D, _D, _D]
        L.ref_orbits_many.argtypes = [ctypes.c_void_p, ctypes.c_long, _D, _D, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_long, _D, _L, _I, ctypes.c_int]
        L.ref_orbits_traj_many.argtypes = [ctypes.c_void_p, ctypes.c_long, _D, _D, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_long, ctypes.c_int, _D, ctypes.c_int]
        L.ref_orbits_evals.argtypes = [ctypes.c_void_p, ctypes.c_long, _D, _D, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_long, _LL, ctypes.c_int]
        L.ref_actions_fd_many.argtypes = [ctypes.c_void_p, ctypes.c_long, _D, _D, _D, _LL, ctypes.c_int]
        L.ref_actions_angles_fd_many.argtypes = [ctypes.c_void_p, ctypes.c_long, _D, _D, _D, _D, _D,
                                                 ctypes.c_int]
        L.ref_actionfinder_create.restype = ctypes.c_void_p
        L.ref_actionfinder_create.argtypes = [ctypes.c_void_p]
        L.ref_actionfinder_free.argtypes = [ctypes.c_void_p]
        L.ref_actionfinder_evalcount.restype = ctypes.c_longlong
        L.ref_actionfinder_evalcount.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_actionfinder_many.argtypes = [ctypes.c_void_p, ctypes.c_long, _D, _D, _D, ctypes.c_int]
        L.ref_actionfinder_table_sizes.argtypes = [ctypes.c_void_p, _L]
        L.ref_actionfinder_tables.argtypes = [ctypes.c_void_p, _D, _D, _D, _D, _D, _D, _D]
        L.ref_actionfinder_lcirc.argtypes = [ctypes.c_void_p, ctypes.c_long, _D, _D]
        _lib = L
    return _lib


def multipole_coefs_from_density(multipole_params, densities):
    """the reference's Multipole::create from the sum of densities (key=value strings), its
    coefficients at full precision: (radii, Phi, dPhi) with Phi, dPhi numCoefs x gridSizeR"""
    L = lib()
    f = L.ref_multipole_from_density
    f.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), _I, _I,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    arr = (ctypes.c_char_p * len(densities))(*[d.encode() for d in densities])
    nr, nc = ctypes.c_int(0), ctypes.c_int(0)
    _check(f(multipole_params.encode(), len(densities), arr, ctypes.byref(nr), ctypes.byref(nc), None, None, None))
    r = np.zeros(nr.value)
    P = np.zeros((nc.value, nr.value))
    D = np.zeros_like(P)
    _check(f(multipole_params.encode(), len(densities), arr, ctypes.byref(nr), ctypes.byref(nc),
             r.ctypes.data, P.ctypes.data, D.ctypes.data))
    return r, P, D


def multipole_potential_from_density(multipole_params, densities):
    """the reference's Multipole from the sum of densities, in memory, as a Potential"""
    L = lib()
    f = L.ref_multipole_potential_from_density
    f.restype = ctypes.c_void_p
    f.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)]
    arr = (ctypes.c_char_p * len(densities))(*[d.encode() for d in densities])
    h = f(multipole_params.encode(), len(densities), arr)
    if not h:
        raise RuntimeError(L.ref_error().decode())
    p = Potential.__new__(Potential)
    p.h = h
    return p


def _p(a, t=_D):
    return None if a is None else a.ctypes.data_as(t)


def _check(rc):
    if rc != 0:
        raise RuntimeError("oracle: " + lib().ref_error().decode())


class Potential:
    """A reference potential, loaded from an INI / coefficient file or key=value parameters."""

    def __init__(self, file=None, params=None):
        L = lib()
        if file is not None:
            self.h = L.ref_load_potential(file.encode())
        else:
            self.h = L.ref_create_potential(params.encode())
        if not self.h:
            raise RuntimeError("oracle: " + L.ref_error().decode())

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.ref_free_potential(self.h)

    def export(self, file):
        _check(lib().ref_write_potential(self.h, file.encode()))

    def eval(self, pos, hess=False, nthreads=0):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        n = len(pos)
        phi = np.empty(n)
        grad = np.empty((n, 3))
        h = np.empty((n, 6)) if hess else None
        _check(lib().ref_eval_many(self.h, n, _p(pos), _p(phi), _p(grad), _p(h), nthreads))
        return (phi, grad, h) if hess else (phi, grad)

    def eval_cyl(self, pos):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        n = len(pos)
        phi, grad, h = np.empty(n), np.empty((n, 3)), np.empty((n, 6))
        _check(lib().ref_eval_cyl_many(self.h, n, _p(pos), _p(phi), _p(grad), _p(h)))
        return phi, grad, h

    def orbits(self, ic, T, Omega=0.0, accuracy=1e-8, maxSteps=0, nthreads=0):
        ic = np.ascontiguousarray(ic, dtype=np.float64).reshape(-1, 6)
        n = len(ic)
        T = np.ascontiguousarray(np.broadcast_to(np.asarray(T, dtype=np.float64), (n,)))
        final = np.empty((n, 6))
        nsteps = np.zeros(n, dtype=np.int64)
        status = np.zeros(n, dtype=np.int32)
        _check(lib().ref_orbits_many(self.h, n, _p(ic), _p(T), Omega, accuracy, maxSteps,
                                     _p(final), _p(nsteps, _L), _p(status, _I), nthreads))
        return final, nsteps, status

    def orbits_traj(self, ic, T, trajsize, Omega=0.0, accuracy=1e-8, maxSteps=0, nthreads=0):
        """trajectories at trajsize regular times from 0 to T (n x trajsize x 6)"""
        ic = np.ascontiguousarray(ic, dtype=np.float64).reshape(-1, 6)
        n = len(ic)
        T = np.ascontiguousarray(np.broadcast_to(np.asarray(T, dtype=np.float64), (n,)))
        out = np.empty((n, trajsize, 6))
        _check(lib().ref_orbits_traj_many(self.h, n, _p(ic), _p(T), Omega, accuracy, maxSteps, int(trajsize),
                                          _p(out), nthreads))
        return out

    def orbit_evals(self, ic, T, Omega=0.0, accuracy=1e-8, maxSteps=0, nthreads=0):
        """potential evaluations spent on each orbit"""
        ic = np.ascontiguousarray(ic, dtype=np.float64).reshape(-1, 6)
        n = len(ic)
        T = np.ascontiguousarray(np.broadcast_to(np.asarray(T, dtype=np.float64), (n,)))
        ev = np.zeros(n, dtype=np.int64)
        _check(lib().ref_orbits_evals(self.h, n, _p(ic), _p(T), Omega, accuracy, maxSteps, _p(ev, _LL), nthreads))
        return ev

    def actions_fd(self, posvel, fd, count=False, nthreads=0):
        posvel = np.ascontiguousarray(posvel, dtype=np.float64).reshape(-1, 6)
        n = len(posvel)
        fd = np.ascontiguousarray(np.broadcast_to(np.asarray(fd, dtype=np.float64), (n,)))
        act = np.empty((n, 3))
        cnt = np.zeros(n, dtype=np.int64) if count else None
        _check(lib().ref_actions_fd_many(self.h, n, _p(posvel), _p(fd), _p(act), _p(cnt, _LL), nthreads))
        return (act, cnt) if count else act

    def actions_angles_fd(self, posvel, fd, nthreads=0):
        posvel = np.ascontiguousarray(posvel, dtype=np.float64).reshape(-1, 6)
        n = len(posvel)
        fd = np.ascontiguousarray(np.broadcast_to(np.asarray(fd, dtype=np.float64), (n,)))
        act, ang, freq = np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
        _check(lib().ref_actions_angles_fd_many(self.h, n, _p(posvel), _p(fd), _p(act), _p(ang),
                                                _p(freq), nthreads))
        return act, ang, freq


class ActionFinder:
    """The reference's ActionFinderAxisymFudge (non-interpolated mode, the default)."""

    def __init__(self, pot):
        self.pot = pot
        self.h = lib().ref_actionfinder_create(pot.h)
        if not self.h:
            raise RuntimeError("oracle: " + lib().ref_error().decode())

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.ref_actionfinder_free(self.h)

    def actions(self, posvel, nthreads=0, with_fd=False):
        posvel = np.ascontiguousarray(posvel, dtype=np.float64).reshape(-1, 6)
        n = len(posvel)
        act = np.empty((n, 3))
        fd = np.empty(n) if with_fd else None
        _check(lib().ref_actionfinder_many(self.h, n, _p(posvel), _p(act), _p(fd), nthreads))
        return (act, fd) if with_fd else act

    def evalcount(self, reset=True):
        return lib().ref_actionfinder_evalcount(self.h, 1 if reset else 0)

    def tables(self):
        sz = np.zeros(5, dtype=np.int64)
        lib().ref_actionfinder_table_sizes(self.h, _p(sz, _L))
        nE, nL, n1, n2, n3 = (int(x) for x in sz)
        gridE, gridL, delta = np.empty(nE), np.empty(nL), np.empty(nE * nL)
        lofe, rofl, phiofr = np.empty(4 * n1), np.empty(4 * n2), np.empty(4 * n3)
        scal = np.empty(5)
        lib().ref_actionfinder_tables(self.h, _p(gridE), _p(gridL), _p(delta), _p(lofe), _p(rofl),
                                      _p(phiofr), _p(scal))
        return dict(gridE=gridE, gridL=gridL, delta=delta.reshape(nE, nL),
                    lofe=lofe.reshape(4, n1), rofl=rofl.reshape(4, n2), phiofr=phiofr.reshape(4, n3),
                    invPhi0=scal[0], interp_invPhi0=scal[1], slopeOut=scal[2], coefOut=scal[3],
                    massOut=scal[4])

    def lcirc(self, E):
        E = np.ascontiguousarray(E, dtype=np.float64)
        L = np.empty_like(E)
        lib().ref_actionfinder_lcirc(self.h, len(E), _p(E), _p(L))
        return L


class CInterfacePotential:
    """A potential through the reference's own plain-C interface (src/interface_c.cpp, compiled
    into the oracle library): agama_createPotential, agama_evalDensity, agama_R_circ,
    agama_R_from_Lz, agama_R_max, agama_findPlanarOrbitExtent, one call per point."""

    def __init__(self, params):
        L = lib()
        L.agama_getError.restype = ctypes.c_char_p
        L.agama_createPotential.restype = ctypes.c_void_p
        L.agama_createPotential.argtypes = [ctypes.c_char_p]
        L.agama_deletePotential.argtypes = [ctypes.c_void_p]
        L.agama_evalDensity.restype = ctypes.c_double
        L.agama_evalDensity.argtypes = [ctypes.c_void_p, _D, ctypes.c_double]
        for name in ("agama_R_circ", "agama_R_from_Lz", "agama_R_max"):
            getattr(L, name).restype = ctypes.c_double
            getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.agama_findPlanarOrbitExtent.restype = None
        L.agama_findPlanarOrbitExtent.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _D, _D]
        self.h = L.agama_createPotential(params.encode())
        if not self.h:
            raise RuntimeError("oracle: " + L.agama_getError().decode())

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.agama_deletePotential(self.h)

    def density(self, pos):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        return np.array([lib().agama_evalDensity(self.h, _p(p), 0.0) for p in pos])

    def R_circ(self, E):
        return np.array([lib().agama_R_circ(self.h, float(e)) for e in np.ravel(E)])

    def R_from_Lz(self, L):
        return np.array([lib().agama_R_from_Lz(self.h, float(x)) for x in np.ravel(L)])

    def R_max(self, E):
        return np.array([lib().agama_R_max(self.h, float(e)) for e in np.ravel(E)])

    def periapo(self, E, L):
        out = np.empty((len(np.ravel(E)), 2))
        r1, r2 = ctypes.c_double(), ctypes.c_double()
        for i, (e, l) in enumerate(zip(np.ravel(E), np.ravel(L))):
            lib().agama_findPlanarOrbitExtent(self.h, float(e), float(l), ctypes.byref(r1), ctypes.byref(r2))
            out[i] = r1.value, r2.value
        return out
