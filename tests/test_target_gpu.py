"""Runtime functions of orbits on the device: the density-grid targets (the reference's
RuntimeFncTarget with TargetDensityClassic<0/1>, src/galaxymodel_target.h:99-150,
src/galaxymodel_densitygrid.cpp:149-238) against the reference's own orbit(..., targets=[...])
on the golden orbits (tests/golden/make_golden.py targets).

Bounds: for regular orbits (as in the orbit parity tests) every recorded value agrees to 1e-6
absolute (the values are time fractions <= 1 stored in FP32; the samples agree to ~1e-9, so a
sample can only change cells within ~1e-9 of a cell boundary); over all orbits the mean fraction of
time inside the grid agrees to 0.02 (chaotic orbits diverge from the reference's); the final
points equal those of the plain orbit batch bit for bit; an orbit of zero time records nothing."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASES = [("cfg1", 0), ("cfg1", 1), ("cfg3", 0)]


@pytest.mark.parametrize("cfg,k", CASES)
def test_density_target_matches_reference(cfg, k):
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "target_%s.npz" % cfg))
    o = np.load(os.path.join(GOLDEN, "orbits_%s.npz" % cfg))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, cfg + ".coef"))
    qy, qz = g["axes%d" % k]
    t = agama_b200.Target(str(g["type%d" % k]), gridr=g["gridr"], stripsPerPane=int(g["strips%d" % k]),
                          axisRatioY=qy, axisRatioZ=qz)
    ref = g["result%d" % k]
    assert len(t) == ref.shape[1]
    Omega = float(g["Omega"])
    final, res = agama_b200.orbit_target(pot, g["ic"], g["T"], t, Omega=Omega, accuracy=float(g["accuracy"]))
    assert res.dtype == np.float32 and res.shape == ref.shape
    plain = agama_b200.orbit(pot, g["ic"], g["T"], Omega=Omega, accuracy=float(g["accuracy"]))
    assert np.array_equal(final, plain)
    reg = o["regular"] & (o["status"] == 0)
    err = np.abs(res[reg] - ref[reg]).max()
    print(cfg, g["type%d" % k], "regular orbits: max |difference| %.3g over %d orbits" % (err, reg.sum()))
    assert err <= 1e-6, err
    # all orbits: the mean fraction of time inside the grid (chaotic orbits diverge from the
    # reference's, so only the set is compared)
    dmean = abs(res.sum(1).mean() - ref.sum(1).mean())
    print(cfg, "all orbits: mean time inside the grid differs by %.3g" % dmean)
    assert dmean <= 0.02
    zero = g["T"] == 0
    assert np.all(res[zero] == 0)


def test_density_target_on_device_buffers():
    import torch
    import agama_b200
    g = np.load(os.path.join(GOLDEN, "target_cfg1.npz"))
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg1.coef"))
    t = agama_b200.Target("DensityClassicTopHat", gridr=g["gridr"], stripsPerPane=2, axisRatioY=0.8, axisRatioZ=0.6)
    f_host, r_host = agama_b200.orbit_target(pot, g["ic"], g["T"], t)
    f_dev, r_dev = agama_b200.orbit_target(pot, torch.tensor(g["ic"], device="cuda"),
                                           torch.tensor(g["T"], device="cuda"), t)
    torch.cuda.synchronize()
    assert np.array_equal(f_dev.cpu().numpy(), f_host) and np.array_equal(r_dev.cpu().numpy(), r_host)
