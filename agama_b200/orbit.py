"""DOP853 orbit integration on the device.

Mirror of the reference's Python orbit() (src/interface_python.cpp:7689-8200) for the
final-point output (trajsize = 1): orbits start at ic (x,y,z,vx,vy,vz in the frame rotating with
pattern speed Omega) at time 0 and are integrated for `time` (scalar or per orbit).
"""
import ctypes

import numpy as np

from . import _native
from ._native import check, ptr


def trajectory(potential, ic, time, trajsize, Omega=0.0, accuracy=1e-8, maxNumSteps=0):
    """Orbits sampled at trajsize regular times from 0 to time (per orbit), as the reference's
    orbit(..., trajsize=N): returns (times n x N, trajectories n x N x 6); numpy in, numpy out."""
    x = np.ascontiguousarray(ic, dtype=np.float64).reshape(-1, 6)
    n = len(x)
    T = np.ascontiguousarray(np.broadcast_to(np.asarray(time, dtype=np.float64), (n,)))
    traj = np.empty((n, int(trajsize), 6))
    check(_native.lib().agama_integrateOrbitsTrajectoryMany(
        potential.handle, n, ptr(x), ptr(T), float(Omega), float(accuracy), int(maxNumSteps), int(trajsize),
        ptr(traj), None, None, None))
    times = T[:, None] * np.linspace(0, 1, int(trajsize))[None, :]
    return times, traj


class Target:
    """A density-grid target for orbits (the reference's Target(type='DensityClassicTopHat' or
    'DensityClassicLinear', gridr=..., stripsPerPane=2, axisRatioY=1, axisRatioZ=1)): radial shells
    with three panes of stripsPerPane^2 cells per octant surface; orbit_target() records, for each
    orbit, the fraction of its time spent in each cell (top-hat) or the trilinear weights of the
    grid nodes (linear)."""

    def __init__(self, type="DensityClassicTopHat", gridr=None, stripsPerPane=2, axisRatioY=1.0, axisRatioZ=1.0):
        t = str(type).lower()
        if t not in ("densityclassictophat", "densityclassiclinear"):
            raise ValueError("Target: only DensityClassicTopHat / DensityClassicLinear are supported")
        g = np.ascontiguousarray(gridr, dtype=np.float64).ravel()
        if len(g) < 2:
            raise ValueError("gridr must be an array with >=2 elements")
        h = _native.lib().agama_createTargetDensityClassic(0 if t.endswith("tophat") else 1, int(stripsPerPane),
                                                           len(g), ptr(g), float(axisRatioY), float(axisRatioZ))
        if not h:
            raise ValueError("agama_b200: " + _native.error())
        self._h = ctypes.c_void_p(h)

    def __len__(self):
        return _native.lib().agama_targetNumCoefs(self._h)

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(_native, "_lib", None)     # module globals may be gone at interpreter exit
        if h and lib is not None:
            lib.agama_deleteTarget(h)
            self._h = None


def orbit_target(potential, ic, time, target, Omega=0.0, accuracy=1e-8, maxNumSteps=0):
    """Orbits with a target's runtime function (as the reference's orbit(..., targets=[target])):
    returns (final points n x 6, n x len(target) float32 matrix of the time-weighted samples of
    each orbit, normalised by its integration time); numpy or CUDA tensors in, the same out."""
    from . import _is_device_array, _dev_ptr, _current_stream
    m = len(target)
    if _is_device_array(ic):
        import torch
        x = ic.contiguous().view(-1, 6)
        n = x.shape[0]
        T = time if _is_device_array(time) else torch.full((n,), float(time), dtype=torch.float64, device=x.device)
        T = T.contiguous()
        out = torch.empty_like(x)
        res = torch.empty((n, m), dtype=torch.float32, device=x.device)
        check(_native.lib().agama_integrateOrbitsTargetManyDevice(
            potential.handle, n, _dev_ptr(x), _dev_ptr(T), float(Omega), float(accuracy), int(maxNumSteps),
            target._h, _dev_ptr(res), _dev_ptr(out), None, None, _current_stream()))
        return out, res
    x = np.ascontiguousarray(ic, dtype=np.float64).reshape(-1, 6)
    n = len(x)
    T = np.ascontiguousarray(np.broadcast_to(np.asarray(time, dtype=np.float64), (n,)))
    out = np.empty((n, 6))
    res = np.empty((n, m), dtype=np.float32)
    check(_native.lib().agama_integrateOrbitsTargetMany(
        potential.handle, n, ptr(x), ptr(T), float(Omega), float(accuracy), int(maxNumSteps), target._h,
        res.ctypes.data_as(_native.F), ptr(out), None, None))
    return out, res


def orbit(potential, ic, time, Omega=0.0, accuracy=1e-8, maxNumSteps=0, queue=True, info=False):
    """Integrate orbits; returns the final phase-space points (n x 6), and with info=True also
    a dict with the accepted step counts, rejected attempts and statuses
    (0 ok, 1 step limit reached, 2 zero / non-finite step, 3 non-finite error estimate).

    ic / time may be numpy arrays (host; copied to the device and back) or CUDA torch tensors
    (processed in place on the current stream; the outputs are then tensors too).
    queue=True drains the batch from a device work queue (best for uneven integration times).
    """
    from . import _is_device_array, _dev_ptr, _current_stream
    if _is_device_array(ic):
        import torch
        x = ic.contiguous().view(-1, 6)
        n = x.shape[0]
        T = time if _is_device_array(time) else torch.full((n,), float(time), dtype=torch.float64, device=x.device)
        T = T.contiguous()
        out = torch.empty_like(x)
        steps = torch.empty(n, dtype=torch.int64, device=x.device)
        rej = torch.empty(n, dtype=torch.int64, device=x.device)
        st = torch.empty(n, dtype=torch.int32, device=x.device)
        check(_native.lib().agama_integrateOrbitsManyDevice(
            potential.handle, n, _dev_ptr(x), _dev_ptr(T), float(Omega), float(accuracy), int(maxNumSteps),
            _dev_ptr(out), _dev_ptr(steps), _dev_ptr(rej), _dev_ptr(st), 1 if queue else 0, _current_stream()))
        return (out, dict(steps=steps, rejected=rej, status=st)) if info else out
    x = np.ascontiguousarray(ic, dtype=np.float64)
    single = x.ndim == 1
    x = x.reshape(-1, 6)
    n = len(x)
    T = np.ascontiguousarray(np.broadcast_to(np.asarray(time, dtype=np.float64), (n,)))
    from . import _host_empty
    out = _host_empty((n, 6))
    steps = _host_empty(n, np.int64)
    st = _host_empty(n, np.int32)
    check(_native.lib().agama_integrateOrbitsMany(
        potential.handle, n, ptr(x), ptr(T), float(Omega), float(accuracy), int(maxNumSteps),
        ptr(out), steps.ctypes.data_as(_native.L), st.ctypes.data_as(_native.I)))
    if single:
        out = out[0]
    return (out, dict(steps=steps, status=st)) if info else out


def set_orbit_precision(mixed=False):
    """mixed=True: later orbit batches in multi-harmonic potentials evaluate the m != 0 harmonics
    of the force in FP32 (radial m = 0 part, azimuthal sums, state, stages and error norm in FP64);
    False (the default): everything in FP64.  jacobi_energy_error() states the error per orbit."""
    check(_native.lib().agama_setOrbitPrecision(1 if mixed else 0))


def jacobi_energy_error(potential, ic, final, Omega=0.0):
    """relative change |E_J(final) / E_J(ic) - 1| of the Jacobi energy
    E_J = Phi + v^2/2 - Omega (x v_y - y v_x) of each orbit, Phi evaluated in FP64: the per-orbit
    error statement of an integration (the integrator's own truncation error plus, in mixed
    precision, the effect of the FP32 harmonics); numpy or CUDA tensors in, the same out."""
    def ej(w):
        phi = potential.potential(w[:, :3])
        return phi + 0.5 * (w[:, 3:] ** 2).sum(1) - Omega * (w[:, 0] * w[:, 4] - w[:, 1] * w[:, 3])
    return abs(ej(final) / ej(ic) - 1)


def set_orbit_lanes(lanes=0):
    """lanes of a warp integrating one orbit together: 1, 2, 4, 8, or 0 (autotuned, the default)"""
    check(_native.lib().agama_setOrbitLanesPerOrbit(int(lanes)))


def set_orbit_block(block=0):
    """threads per block of the orbit kernels: 32, 64, 128, or 0 (autotuned with the lanes, the
    default); no setting changes a result"""
    check(_native.lib().agama_setOrbitBlockSize(int(block)))


class OrbitGraph:
    """an orbit batch over CUDA tensors captured once in a CUDA graph; launch() replays it on the
    current stream (with final is ic, every launch continues the orbits for another T)"""

    def __init__(self, potential, ic, time, Omega=0.0, accuracy=1e-8, maxNumSteps=0, final=None):
        import torch
        from . import _dev_ptr
        self.potential = potential
        self.ic = ic
        n = ic.shape[0]
        self.T = time if hasattr(time, "data_ptr") else torch.full((n,), float(time), dtype=torch.float64,
                                                                    device=ic.device)
        self.final = torch.empty_like(ic) if final is None else final
        self.steps = torch.empty(n, dtype=torch.int64, device=ic.device)
        self.rejected = torch.empty(n, dtype=torch.int64, device=ic.device)
        self.status = torch.empty(n, dtype=torch.int32, device=ic.device)
        h = _native.lib().agama_orbitGraphCreate(potential.handle, n, _dev_ptr(ic), _dev_ptr(self.T), float(Omega),
                                                 float(accuracy), int(maxNumSteps), _dev_ptr(self.final),
                                                 _dev_ptr(self.steps), _dev_ptr(self.rejected), _dev_ptr(self.status))
        if not h:
            raise RuntimeError("agama_b200: " + _native.error())
        self._h = ctypes.c_void_p(h)

    @property
    def lanes(self):
        return _native.lib().agama_orbitGraphLanes(self._h)

    @property
    def block(self):
        return _native.lib().agama_orbitGraphBlockSize(self._h)

    def launch(self):
        from . import _current_stream
        check(_native.lib().agama_orbitGraphLaunch(self._h, _current_stream()))
        return self.final

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(_native, "_lib", None)     # module globals may be gone at interpreter exit
        if h and lib is not None:
            lib.agama_orbitGraphDelete(h)
            self._h = None
