"""Staeckel-fudge action finder on the device.

Mirror of the reference's Python ActionFinder / actions (src/interface_python.cpp:3705-3860):

    af = ActionFinder(potential, tables=...)     # focal-distance table + L_circ(E) interpolator
    J  = af(points)                              # (n, 3): Jr, Jz, Jphi
    J  = actions(potential, points, fd=...)      # fixed focal distance(s)
    J, theta, Omega = af(points, angles=True, frequencies=True)

`points` are Cartesian phase-space points (n x 6) as numpy arrays (host) or CUDA torch tensors
(device, processed on the current stream).
"""
import ctypes

import numpy as np

from . import _native
from ._native import check, ptr


def _host_empty(shape):
    from . import _host_empty as he
    return he(shape)


class ActionFinder:
    """Staeckel-fudge action finder (the reference's ActionFinderAxisymFudge, non-interpolated).

    tables: dict with gridE, gridL, delta (nE x nL), lofe / rofl / phiofr (4 x n: x, f, f', f''),
    invPhi0, interp_invPhi0, slopeOut, coefOut, massOut -- the focal-distance grid and the
    L_circ(E) interpolator of the finder.
    """

    def __init__(self, potential, tables=None):
        self.potential = potential
        if tables is None:
            # build the focal-distance table (shell orbits on the device) and L_circ(E)
            h = _native.lib().agama_createActionFinder(potential.handle)
            if not h:
                raise RuntimeError("agama_b200: " + _native.error())
            self._h = ctypes.c_void_p(h)
            return
        t = {k: np.ascontiguousarray(v, dtype=np.float64) if isinstance(v, np.ndarray) else v
             for k, v in tables.items()}
        gE, gL, dl = t["gridE"], t["gridL"], np.ascontiguousarray(t["delta"], dtype=np.float64)
        lofe, rofl, phr = (np.ascontiguousarray(t[k], dtype=np.float64) for k in ("lofe", "rofl", "phiofr"))
        scal = np.array([t["invPhi0"], t["interp_invPhi0"], t["slopeOut"], t["coefOut"], t["massOut"]], dtype=np.float64)
        h = _native.lib().agama_createActionFinderFromTables(
            potential.handle, len(gE), ptr(gE), len(gL), ptr(gL), ptr(dl), lofe.shape[1], ptr(lofe),
            rofl.shape[1], ptr(rofl), phr.shape[1], ptr(phr), ptr(scal))
        if not h:
            raise RuntimeError("agama_b200: " + _native.error())
        self._h = ctypes.c_void_p(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(_native, "_lib", None)     # module globals may be gone at interpreter exit
        if h and lib is not None:
            lib.agama_deleteActionFinder(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def tables(self):
        """the finder's tables, in the layout accepted by ActionFinder(potential, tables=...)"""
        L = _native.lib()
        sz = [ctypes.c_int() for _ in range(5)]
        check(L.agama_getActionFinderTableSizes(self._h, *[ctypes.byref(x) for x in sz]))
        nE, nL, n1, n2, n3 = (x.value for x in sz)
        gE, gL, dl = np.empty(nE), np.empty(nL), np.empty((nE, nL))
        lofe, rofl, phr, scal = np.empty((4, n1)), np.empty((4, n2)), np.empty((4, n3)), np.empty(5)
        check(L.agama_getActionFinderTables(self._h, ptr(gE), ptr(gL), ptr(dl), ptr(lofe), ptr(rofl), ptr(phr),
                                            ptr(scal)))
        return dict(gridE=gE, gridL=gL, delta=dl, lofe=lofe, rofl=rofl, phiofr=phr, invPhi0=scal[0],
                    interp_invPhi0=scal[1], slopeOut=scal[2], coefOut=scal[3], massOut=scal[4])

    # ---- learned root brackets
    def bracket_samples(self, points):
        """inputs (n x 6), targets (n x 3) and masks (n x 3) of the bracket predictor from the plain
        root searches of the points"""
        p = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 6)
        n = len(p)
        f, t, m = (np.empty((n, k), dtype=np.float32) for k in (6, 3, 3))
        check(_native.lib().agama_actionFinderBracketSamples(self._h, n, ptr(p), ptr(f, _native.F), ptr(t, _native.F),
                                                             ptr(m, _native.F)))
        return f, t, m

    def train_brackets(self, points, epochs=10, batch=2048, lr=2e-3, seed=0):
        """train the bracket predictor on the finder's own root searches for these points and
        switch it on; returns (loss per epoch, bracket half-widths)"""
        p = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 6)
        hist, w = np.empty(epochs, dtype=np.float32), np.empty(3, dtype=np.float32)
        check(_native.lib().agama_actionFinderTrainBrackets(self._h, len(p), ptr(p), int(epochs), int(batch), float(lr),
                                                            int(seed), ptr(hist, _native.F), ptr(w, _native.F)))
        return hist, w

    def predict_brackets(self, features):
        """the trained network's predictions (n x 3) for inputs as returned by bracket_samples"""
        f = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, 6)
        y = np.empty((len(f), 3), dtype=np.float32)
        check(_native.lib().agama_actionFinderPredictBrackets(self._h, len(f), ptr(f, _native.F), ptr(y, _native.F)))
        return y

    def use_brackets(self, on=True):
        check(_native.lib().agama_actionFinderUseBrackets(self._h, 1 if on else 0))

    def count_brackets(self, on=True):
        """keep (True, the default) or stop the root-search counters of bracket_stats(); without
        them the searches run in a kernel compiled without the counters"""
        check(_native.lib().agama_actionFinderCountBrackets(self._h, 1 if on else 0))

    def bracket_stats(self, reset=False):
        """{searches, narrowed, fallbacks, iterations} of the root searches since the last reset:
        narrowed = searches started from a predicted root, fallbacks = plain searches after a
        failed check of such a root"""
        st = (ctypes.c_longlong * 4)()
        check(_native.lib().agama_actionFinderBracketStats(self._h, st, 1 if reset else 0))
        return dict(searches=st[0], narrowed=st[1], fallbacks=st[2], iterations=st[3])

    def __call__(self, points, fd=False, actions=True, angles=False, frequencies=False):
        """actions (n x 3: Jr, Jz, Jphi); with fd=True also the focal distance used for each point.
        With angles / frequencies (n x 3: theta_r, theta_z, theta_phi / Omega_r, Omega_z,
        Omega_phi), the requested arrays come back as a tuple in the order actions, angles,
        frequencies, as the reference's ActionFinder does."""
        from . import _is_device_array, _dev_ptr, _current_stream
        if angles or frequencies:
            if fd:
                raise ValueError("fd=True is not combined with angles / frequencies")
            return _angles_call(points, actions, angles, frequencies,
                                lambda n, p, a, t, f, dev: (
                                    _native.lib().agama_evalActionsAnglesFrequenciesManyDevice(
                                        self._h, n, p, a, t, f, _current_stream()) if dev else
                                    _native.lib().agama_evalActionsAnglesFrequenciesMany(self._h, n, p, a, t, f)))
        if _is_device_array(points):
            import torch
            p = points.contiguous().view(-1, 6)
            n = p.shape[0]
            act = torch.empty((n, 3), dtype=torch.float64, device=p.device)
            fdo = torch.empty(n, dtype=torch.float64, device=p.device) if fd else None
            check(_native.lib().agama_evalActionsManyDevice(self._h, n, _dev_ptr(p), _dev_ptr(act), _dev_ptr(fdo),
                                                            _current_stream()))
            return (act, fdo) if fd else act
        p = np.ascontiguousarray(points, dtype=np.float64)
        single = p.ndim == 1
        p = p.reshape(-1, 6)
        n = len(p)
        act = _host_empty((n, 3))
        fdo = _host_empty(n) if fd else None
        check(_native.lib().agama_evalActionsMany(self._h, n, ptr(p), ptr(act), ptr(fdo)))
        if single:
            act = act[0]
        return (act, fdo) if fd else act


def _angles_call(points, want_act, want_ang, want_freq, call):
    """run one of the angle / frequency entry points on host arrays or CUDA tensors"""
    from . import _is_device_array, _dev_ptr
    if _is_device_array(points):
        import torch
        p = points.contiguous().view(-1, 6)
        n = p.shape[0]
        outs = [torch.empty((n, 3), dtype=torch.float64, device=p.device) if w else None
                for w in (want_act, want_ang, want_freq)]
        check(call(n, _dev_ptr(p), *[_dev_ptr(o) for o in outs], True))
        single = False
    else:
        p = np.ascontiguousarray(points, dtype=np.float64)
        single = p.ndim == 1
        p = p.reshape(-1, 6)
        n = len(p)
        outs = [_host_empty((n, 3)) if w else None for w in (want_act, want_ang, want_freq)]
        check(call(n, ptr(p), *[ptr(o) for o in outs], False))
        if single:
            outs = [o[0] if o is not None else None for o in outs]
    res = [o for o in outs if o is not None]
    return res[0] if len(res) == 1 else tuple(res)


def actions(potential, points, fd, iters=False, angles=False, frequencies=False):
    """Staeckel-fudge actions for given focal distance(s) fd (scalar or per point); with angles /
    frequencies the tuple (actions, angles?, frequencies?) as in ActionFinder.__call__."""
    from . import _is_device_array, _dev_ptr, _current_stream
    if angles or frequencies:
        if iters:
            raise ValueError("iters=True is not combined with angles / frequencies")
        if _is_device_array(points):
            fda = fd.contiguous() if _is_device_array(fd) else None
            fdp, fd0 = _dev_ptr(fda), (0.0 if fda is not None else float(fd))
        elif np.ndim(fd) == 0:
            fda, fdp, fd0 = None, None, float(fd)
        else:
            n = len(np.reshape(points, (-1, 6)))
            fda = np.ascontiguousarray(np.broadcast_to(np.asarray(fd, dtype=np.float64), (n,)))
            fdp, fd0 = ptr(fda), 0.0
        return _angles_call(points, True, angles, frequencies,
                            lambda n, p, a, t, f, dev: (
                                _native.lib().agama_evalActionsAnglesFrequenciesStandaloneManyDevice(
                                    potential.handle, n, p, fdp, fd0, a, t, f, _current_stream()) if dev else
                                _native.lib().agama_evalActionsAnglesFrequenciesStandaloneMany(
                                    potential.handle, n, p, fdp, fd0, a, t, f)))
    if _is_device_array(points):
        import torch
        p = points.contiguous().view(-1, 6)
        n = p.shape[0]
        act = torch.empty((n, 3), dtype=torch.float64, device=p.device)
        it = torch.empty(n, dtype=torch.int32, device=p.device) if iters else None
        fda = fd.contiguous() if _is_device_array(fd) else None
        check(_native.lib().agama_evalActionsStandaloneManyDevice(
            potential.handle, n, _dev_ptr(p), _dev_ptr(fda), 0.0 if fda is not None else float(fd),
            _dev_ptr(act), _dev_ptr(it), _current_stream()))
        return (act, it) if iters else act
    p = np.ascontiguousarray(points, dtype=np.float64)
    single = p.ndim == 1
    p = p.reshape(-1, 6)
    n = len(p)
    act = _host_empty((n, 3))
    if np.ndim(fd) == 0:
        check(_native.lib().agama_evalActionsStandaloneMany(potential.handle, n, ptr(p), None, float(fd), ptr(act)))
    else:
        fda = np.ascontiguousarray(np.broadcast_to(np.asarray(fd, dtype=np.float64), (n,)))
        check(_native.lib().agama_evalActionsStandaloneMany(potential.handle, n, ptr(p), ptr(fda), 0.0, ptr(act)))
    return act[0] if single else act


def set_action_precision(mixed=False):
    """mixed=True: later action computations (without angles / frequencies) evaluate the action
    integrands after F(tau) and their Gauss-Legendre sums in FP32 (compensated sums), with the
    potential, F(tau), the integrals of motion and the root searches in FP64; False (the default):
    everything in FP64"""
    check(_native.lib().agama_setActionPrecision(1 if mixed else 0))
