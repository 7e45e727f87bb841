"""agama_b200: a B200-native engine for Agama's orbit-and-action hot path.

Python mirror of the parts of the reference's Python interface (src/interface_python.cpp) that
sit on this path:

    Potential(file=...) / Potential(type='Multipole', file=...)      agama.Potential
        .potential(points), .force(points), .forceDeriv(points), .eval(...)
    ActionFinder(potential)(points)                                   agama.ActionFinder
    actions(potential, points, fd=...)                                agama.actions
    orbit(potential=..., ic=..., time=..., Omega=..., accuracy=...)   agama.orbit

Inputs may be numpy arrays (host; copied to the device and back) or CUDA tensors exposing
__cuda_array_interface__ / torch tensors (device; processed in place on the current stream).
All computation runs in the CUDA kernels of libagama_b200.so -- there is no CPU fallback.
"""
import ctypes

import numpy as np

from . import _native
from ._native import check, ptr

__all__ = ["Potential", "ActionFinder", "actions", "orbit"]


def _is_device_array(a):
    return hasattr(a, "__cuda_array_interface__") or (hasattr(a, "is_cuda") and a.is_cuda)


def _dev_ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return ctypes.c_void_p(a.__cuda_array_interface__["data"][0])


def _current_stream():
    try:
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    except Exception:
        return None


def _host_empty(shape, dtype=np.float64):
    """a host output array in page-locked memory (torch's caching host allocator, so repeated
    calls reuse the same blocks) when CUDA is usable: device-to-host copies into it run at full
    PCIe speed and overlap the kernels of the next chunk; plain numpy memory otherwise"""
    try:
        import torch
        if torch.cuda.is_available():
            tdt = {np.float64: torch.float64, np.int64: torch.int64, np.int32: torch.int32}[np.dtype(dtype).type]
            return torch.empty(shape, dtype=tdt, pin_memory=True).numpy()
    except Exception:
        pass
    return np.empty(shape, dtype=dtype)


def _points(a, ncol):
    a = np.ascontiguousarray(a, dtype=np.float64)
    single = a.ndim == 1
    a = a.reshape(-1, ncol)
    return a, single


def _key_values(d):
    """a dict of parameters as the reference's key=value string"""
    return ", ".join("%s=%s" % (k, repr(float(v)) if isinstance(v, float) else v) for k, v in d.items())


def multipole_coefs_from_density(density, **params):
    """the coefficients (radii, Phi, dPhi; Phi and dPhi numCoefs x gridSizeR) of the Multipole that
    Potential(type='Multipole', density=..., **params) builds, computed on the host (no device)"""
    comps = density if isinstance(density, (list, tuple)) else [density]
    dens = (ctypes.c_char_p * len(comps))(*[_key_values(d).encode() for d in comps])
    L = _native.lib()
    nr, nc = ctypes.c_int(0), ctypes.c_int(0)
    mp = _key_values(params).encode()
    check(L.agama_multipoleCoefsFromDensities(mp, len(comps), dens, ctypes.byref(nr), ctypes.byref(nc), None, None,
                                              None))
    r = np.zeros(nr.value)
    P = np.zeros((nc.value, nr.value))
    D = np.zeros_like(P)
    check(L.agama_multipoleCoefsFromDensities(mp, len(comps), dens, ctypes.byref(nr), ctypes.byref(nc),
                                              ptr(r), ptr(P), ptr(D)))
    return r, P, D


class Potential:
    """A Multipole potential resident on the current CUDA device.

    Potential(file='coefs.ini')                     -- coefficient file of the reference format
    Potential(type='Multipole', file='coefs.ini')
    Potential(radii=r, Phi=P, dPhi=dP)              -- arrays as in Multipole(gridRadii, Phi, dPhi)
    Potential(type='Multipole', density=dict(type='Dehnen', mass=1, ...), lmax=6, gridSizeR=50, ...)
                                                    -- the Poisson solve from a density model (or a
                                                       list of them, summed), as the reference's
                                                       Potential(type='Multipole', density=...)
    """

    def __init__(self, file=None, type="Multipole", radii=None, Phi=None, dPhi=None, density=None, **params):
        L = _native.lib()
        if density is not None:
            comps = density if isinstance(density, (list, tuple)) else [density]
            dens = (ctypes.c_char_p * len(comps))(*[_key_values(d).encode() for d in comps])
            h = L.agama_createMultipoleFromDensities(_key_values(params).encode(), len(comps), dens)
        elif file is not None:
            params = "type=%s, file=%s" % (type, file)
            h = L.agama_createPotential(params.encode())
        elif radii is not None:
            radii = np.ascontiguousarray(radii, dtype=np.float64)
            Phi = np.ascontiguousarray(Phi, dtype=np.float64)
            dPhi = np.ascontiguousarray(dPhi, dtype=np.float64)
            if Phi.shape != dPhi.shape or Phi.shape[1] != len(radii):
                raise ValueError("Phi and dPhi must have shape (numCoefs, len(radii))")
            h = L.agama_createMultipoleFromCoefs(len(radii), ptr(radii), Phi.shape[0], ptr(Phi), ptr(dPhi))
        else:
            raise ValueError("Potential: give file=... or radii/Phi/dPhi arrays")
        if not h:
            raise RuntimeError("agama_b200: " + _native.error())
        self._h = ctypes.c_void_p(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(_native, "_lib", None)     # module globals may be gone at interpreter exit
        if h and lib is not None:
            lib.agama_deletePotential(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def info(self):
        v = [ctypes.c_int() for _ in range(5)]
        check(_native.lib().agama_getPotentialInfo(self._h, *[ctypes.byref(x) for x in v]))
        lmax, mmax, sym, nr, nt = (x.value for x in v)
        return dict(lmax=lmax, mmax=mmax, symmetry=sym, gridSizeR=nr, gridSizeTau=nt)

    def export(self, file):
        """write the coefficient file of this potential (the reference's Potential.export /
        writePotential text format, numbers with 17 significant digits), readable by the reference
        and by Potential(file=...)"""
        check(_native.lib().agama_writePotential(str(file).encode(), self._h))

    # ---------------- evaluation ----------------
    def eval(self, points, pot=True, acc=False, der=False):
        """Potential, acceleration (-grad Phi) and/or Hessian (xx,yy,zz,xy,yz,zx) at points."""
        if _is_device_array(points):
            return self._eval_device(points, pot, acc, der)
        p, single = _points(points, 3)
        n = len(p)
        phi = _host_empty(n)
        grad = _host_empty((n, 3)) if (acc or der) else None
        hess = _host_empty((n, 6)) if der else None
        check(_native.lib().agama_evalPotentialMany(self._h, n, ptr(p), 0.0, ptr(phi), ptr(grad), ptr(hess)))
        out = []
        if pot:
            out.append(phi[0] if single else phi)
        if acc:
            out.append(-grad[0] if single else -grad)
        if der:
            out.append(hess[0] if single else hess)
        return out[0] if len(out) == 1 else tuple(out)

    def _eval_device(self, points, pot, acc, der):
        import torch
        p = points.contiguous().view(-1, 3)
        n = p.shape[0]
        phi = torch.empty(n, dtype=torch.float64, device=p.device)
        grad = torch.empty((n, 3), dtype=torch.float64, device=p.device) if (acc or der) else None
        hess = torch.empty((n, 6), dtype=torch.float64, device=p.device) if der else None
        check(_native.lib().agama_evalPotentialManyDevice(
            self._h, n, _dev_ptr(p), _dev_ptr(phi), _dev_ptr(grad), _dev_ptr(hess), _current_stream()))
        out = []
        if pot:
            out.append(phi)
        if acc:
            out.append(-grad)
        if der:
            out.append(hess)
        return out[0] if len(out) == 1 else tuple(out)

    def eval_cyl(self, points):
        """potential, gradient (dR, dz, dphi) and Hessian (dR2, dz2, dphi2, dRdz, dzdphi, dRdphi) at
        cylindrical points (R, z, phi), evaluated in cylindrical coordinates as the reference's
        BasePotential::eval(PosCyl, ...) (host arrays)"""
        p, single = _points(points, 3)
        n = len(p)
        phi, grad, hess = _host_empty(n), _host_empty((n, 3)), _host_empty((n, 6))
        check(_native.lib().agama_evalPotentialCylMany(self._h, n, ptr(p), 0.0, ptr(phi), ptr(grad), ptr(hess)))
        return (phi[0], grad[0], hess[0]) if single else (phi, grad, hess)

    def potential(self, points):
        return self.eval(points, pot=True)

    def force(self, points):
        return self.eval(points, pot=False, acc=True)

    def forceDeriv(self, points):
        """force and the derivatives of force (= minus the Hessian), as agama's forceDeriv"""
        f, h = self.eval(points, pot=False, acc=True, der=True)
        return f, -h

    def density(self, points):
        """density (Laplacian of the potential / 4 pi) at points, as agama's Potential.density"""
        if _is_device_array(points):
            import torch
            p = points.contiguous().view(-1, 3)
            rho = torch.empty(p.shape[0], dtype=torch.float64, device=p.device)
            check(_native.lib().agama_evalDensityManyDevice(self._h, p.shape[0], _dev_ptr(p), _dev_ptr(rho),
                                                            _current_stream()))
            return rho
        p, single = _points(points, 3)
        rho = _host_empty(len(p))
        check(_native.lib().agama_evalDensityMany(self._h, len(p), ptr(p), 0.0, ptr(rho)))
        return rho[0] if single else rho

    # ---------------- radii in the equatorial plane (azimuthally averaged potential) ----------------
    def _radii(self, query, a, b=None):
        a = np.ascontiguousarray(a, dtype=np.float64)
        single = a.ndim == 0
        a = a.reshape(-1)
        n = len(a)
        out1 = _host_empty(n)
        out2 = _host_empty(n) if b is not None else None
        if b is not None:
            b = np.ascontiguousarray(np.broadcast_to(np.asarray(b, dtype=np.float64).reshape(-1), (n,)))
        check(_native.lib().agama_potentialRadiiMany(self._h, query, n, ptr(a), ptr(b), ptr(out1), ptr(out2)))
        if b is None:
            return out1[0] if single else out1
        res = np.column_stack([out1, out2])
        return res[0] if single else res

    def Rcirc(self, L=None, E=None):
        """radius of the circular orbit with angular momentum L or energy E (exactly one of them),
        as agama's Potential.Rcirc (potential::R_from_Lz / R_circ)"""
        if (L is None) == (E is None):
            raise TypeError("Rcirc() takes exactly one argument (either L or E)")
        return self._radii(1, L) if L is not None else self._radii(0, E)

    def Rmax(self, E):
        """root of Phi(R, z = 0) = E (potential::R_max)"""
        return self._radii(2, E)

    def Rperiapo(self, EL):
        """peri- and apocentre radii of planar orbits from (E, L) pairs, as agama's Potential.Rperiapo
        (potential::findPlanarOrbitExtent); returns (Rperi, Rapo) or an N x 2 array"""
        EL = np.asarray(EL, dtype=np.float64)
        if EL.shape[-1] != 2:
            raise ValueError("Rperiapo: input must be a pair (E, L) or an N x 2 array of them")
        if EL.ndim == 1:
            return self._radii(3, EL[0], EL[1])
        return self._radii(3, EL[:, 0], EL[:, 1])


from .actions import ActionFinder, actions, set_action_precision  # noqa: E402,F401
from .orbit import (orbit, orbit_target, Target, set_orbit_lanes, set_orbit_block, set_orbit_precision, jacobi_energy_error,  # noqa: E402,F401
                    trajectory, OrbitGraph)
from .mlp import BracketNet  # noqa: E402,F401
