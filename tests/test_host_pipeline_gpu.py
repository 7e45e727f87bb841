"""Host-buffer batches are cut into chunks that overlap copies with kernels; their results must
equal those of one device-pointer launch bit for bit, for pinned and pageable host arrays, with
ragged last chunks and optional outputs left out; batches of at least 524 288 items take five
growing chunks, smaller ones four equal chunks."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _points(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, 3)) * np.exp(rng.uniform(-3, 3, (n, 1)))
    return np.ascontiguousarray(x)


@pytest.mark.parametrize("n", [65536 * 3 + 17, 1000003])
def test_potential_host_chunks_equal_device(n):
    import torch
    import agama_b200
    from agama_b200 import _native
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg1.coef"))
    x = _points(n, 11)
    phi_h, acc_h, der_h = pot.eval(x, pot=True, acc=True, der=True)
    xd = torch.tensor(x, device="cuda")
    phi_d, acc_d, der_d = pot.eval(xd, pot=True, acc=True, der=True)
    torch.cuda.synchronize()
    assert np.array_equal(phi_h, phi_d.cpu().numpy())
    assert np.array_equal(acc_h, acc_d.cpu().numpy())
    assert np.array_equal(der_h, der_d.cpu().numpy())
    # pinned input, only the gradient requested (the gradient-only kernel is a different
    # instantiation from the one with the Hessian: compare with its device launch)
    xp = torch.from_numpy(x).pin_memory()
    g = np.empty((n, 3))
    _native.check(_native.lib().agama_evalPotentialMany(pot.handle, n, _native.ptr(xp.numpy()), 0.0, None,
                                                        _native.ptr(g), None))
    acc_only = pot.force(xd)
    torch.cuda.synchronize()
    assert np.array_equal(-g, acc_only.cpu().numpy())
    assert np.allclose(-g, acc_h, rtol=1e-13, atol=1e-15 * np.max(np.abs(acc_h)))


@pytest.mark.parametrize("n", [65536 * 2 + 5, 600001])
def test_actions_host_chunks_equal_device(n):
    """n = 600001: the five growing chunks of large batches (5 % ... 10 % of the batch)"""
    import torch
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "actions_cfg2.npz"))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg2.coef"))
    af = agama_b200.ActionFinder(pot)
    base = g["points"]
    reps = n // len(base) + 1
    rng = np.random.default_rng(3)
    pts = np.ascontiguousarray(np.tile(base, (reps, 1)) * (1 + 1e-3 * rng.standard_normal((reps * len(base), 6))))
    J_h, fd_h = af(pts, fd=True)
    J_d, fd_d = af(torch.tensor(pts, device="cuda"), fd=True)
    torch.cuda.synchronize()
    assert np.array_equal(J_h, J_d.cpu().numpy(), equal_nan=True)
    assert np.array_equal(fd_h, fd_d.cpu().numpy(), equal_nan=True)
    # fixed focal distance per point (a second per-item input)
    fd = np.abs(fd_h) + 0.1
    fd[~np.isfinite(fd)] = 1.0
    Js_h = agama_b200.actions(pot, pts, fd=fd)
    Js_d = agama_b200.actions(pot, torch.tensor(pts, device="cuda"), fd=torch.tensor(fd, device="cuda"))
    torch.cuda.synchronize()
    assert np.array_equal(Js_h, Js_d.cpu().numpy(), equal_nan=True)
