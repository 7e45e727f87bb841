"""The allocation-free orbit entry point (agama_integrateOrbitsManyDeviceNoAlloc).

It serves callers that cannot let a library allocate device memory (an application whose
memory manager already holds the GPU's memory, latency-critical loops where an allocation would
synchronise the device, plugin hosts that account for all device memory).  Its work-queue counter
sits in a static device array of 32 slots instead of a per-call allocation.

Checked here, through the C-ABI: two calls in a row give the same final points, step counts and
statuses as the allocating entry point (agama_integrateOrbitsManyDevice with the work queue, one
lane per orbit as the allocation-free call uses), within the orbit tests' bound of 1e-7 (the second
call shows that the counter is cleared between calls); the device's free memory is the same before
and after a call (nothing was allocated; the first call may load the kernel's code, so this is
checked on the second); an out-of-range slot is rejected with an error.  This file is collected
last.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _buffers(ic):
    import torch
    n = ic.shape[0]
    return (torch.empty_like(ic), torch.empty(n, dtype=torch.int64, device=ic.device),
            torch.empty(n, dtype=torch.int64, device=ic.device), torch.empty(n, dtype=torch.int32, device=ic.device))


def _run(pot, ic, T, bufs, slot=None):
    """one batch through the C-ABI into preallocated buffers; slot None: the allocating entry point"""
    import torch
    from agama_b200 import _native, _dev_ptr
    out, steps, rej, st = bufs
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = [pot.handle, ic.shape[0], _dev_ptr(ic), _dev_ptr(T), 0.0, 1e-8, 0, _dev_ptr(out), _dev_ptr(steps),
            _dev_ptr(rej), _dev_ptr(st)]
    lib = _native.lib()
    if slot is None:
        rc = lib.agama_integrateOrbitsManyDevice(*args, 1, stream)
    else:
        rc = lib.agama_integrateOrbitsManyDeviceNoAlloc(*args, slot, stream)
    assert rc == 0, _native.error()
    torch.cuda.synchronize()


def _host(bufs):
    return tuple(b.cpu().numpy() for b in bufs)


def test_no_alloc_orbits_match_allocating_entry_point():
    import torch
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "orbits_cfg1.npz"))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg1.coef"))
    ic = torch.tensor(g["ic"], device="cuda")
    T = torch.tensor(g["T"], device="cuda")
    ref_bufs = _buffers(ic)
    agama_b200.set_orbit_lanes(1)          # the allocation-free call runs one lane per orbit
    try:
        _run(pot, ic, T, ref_bufs)
    finally:
        agama_b200.set_orbit_lanes(0)
    ref_out, ref_steps, ref_rej, ref_st = _host(ref_bufs)
    bufs = _buffers(ic)
    for call in range(2):          # two calls in a row: the shared counter must be cleared each time
        bufs[0].fill_(np.nan)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        _run(pot, ic, T, bufs, slot=3)
        free_after = torch.cuda.mem_get_info()[0]
        if call == 1:
            assert free_after == free_before, (free_before, free_after)
        out, steps, rej, st = _host(bufs)
        scale = np.maximum(np.linalg.norm(ref_out[:, :3], axis=1), 1e-300)
        assert np.all(np.linalg.norm(out[:, :3] - ref_out[:, :3], axis=1) <= 1e-7 * scale), call
        vscale = np.maximum(np.linalg.norm(ref_out[:, 3:], axis=1), 1e-300)
        assert np.all(np.linalg.norm(out[:, 3:] - ref_out[:, 3:], axis=1) <= 1e-7 * vscale), call
        assert np.array_equal(steps, ref_steps) and np.array_equal(st, ref_st), call
        assert np.array_equal(rej, ref_rej), call


def test_no_alloc_rejects_bad_slot():
    import torch
    import agama_b200
    from agama_b200 import _native, _dev_ptr
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg1.coef"))
    ic = torch.zeros((4, 6), dtype=torch.float64, device="cuda")
    T = torch.ones(4, dtype=torch.float64, device="cuda")
    out = torch.empty_like(ic)
    for slot in (-1, 32):
        rc = _native.lib().agama_integrateOrbitsManyDeviceNoAlloc(
            pot.handle, 4, _dev_ptr(ic), _dev_ptr(T), 0.0, 1e-8, 0, _dev_ptr(out), None, None, None, slot, None)
        assert rc != 0 and "queueSlot" in _native.error()
