"""Learned root brackets of the action finder (the config-4 form: the config-1 potential made
axisymmetric, trained on its own distribution): the network is trained on the finder's own root
searches, the searches take its predicted roots as their first iterates inside the plain brackets
and hand a limit to the plain search when the check of its root fails.  The actions must stay
those of the plain searches (1e-6) and of the reference (golden vectors), and the network must
save root-finder iterations."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from test_actions_gpu import check_actions

pytestmark = pytest.mark.gpu


def _config1_points(n, seed):
    import agama_b200
    from agama_b200 import workloads
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg4.coef"))
    pos = workloads.dehnen_positions(n, 1.0, q=(0.8, 0.6), seed=seed)
    return pot, workloads.orbit_ics(pos, pot.potential, seed=seed + 1000)


def test_learned_brackets_keep_the_actions_and_save_iterations():
    """the config-4 protocol of bench.py: trained on 2e6 points, checked on 1e7 others"""
    import torch
    import agama_b200
    from agama_b200 import workloads
    seed = workloads.SEEDS["particles4"]
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg4.coef"))
    pos = workloads.dehnen_positions(2000000, 1.0, q=(0.8, 0.6), seed=seed)
    train = workloads.orbit_ics(pos, pot.potential, seed=seed + 1000)
    pos = workloads.dehnen_positions(10000000, 1.0, q=(0.8, 0.6), seed=seed + 1)
    evalpts = torch.tensor(workloads.orbit_ics(pos, pot.potential, seed=seed + 2000), device="cuda")
    del pos
    af = agama_b200.ActionFinder(pot)
    hist, widths = af.train_brackets(train, epochs=20, batch=2048, lr=2e-3, seed=1)
    print('loss per epoch', hist)
    assert hist[-1] < 0.2 * hist[0], hist
    af.use_brackets(False)
    af.bracket_stats(reset=True)
    J0 = af(evalpts)
    plain = af.bracket_stats(reset=True)
    af.use_brackets(True)
    J1 = af(evalpts)
    learned = af.bracket_stats(reset=True)
    print("bracket half-widths", widths, "loss", hist[0], "->", hist[-1])
    print("plain", plain, "learned", learned)
    J0, J1 = J0.cpu().numpy(), J1.cpu().numpy()
    ok = np.all(np.isfinite(J0), axis=1)
    bad = np.flatnonzero(ok)[np.any(np.abs(J1[ok] - J0[ok]) > 1e-6 * np.abs(J0[ok]) +
                                    1e-9 * np.sum(np.abs(J0[ok]), axis=1, keepdims=True), axis=1)]
    print("points off the plain form:", len(bad), evalpts[bad[:5]].cpu().numpy() if len(bad) else "")
    check_actions(J1, J0)
    # the network saves root-finder iterations (the count includes the one checking evaluation
    # of every search started from a predicted root): a large share of the searches start from
    # its predictions, a few percent of their roots fail the check and go to the plain search
    assert learned["searches"] == plain["searches"] and learned["narrowed"] > 0.3 * learned["searches"]
    assert learned["fallbacks"] < 0.03 * learned["narrowed"]
    assert learned["iterations"] < 0.97 * plain["iterations"]        # measured on B200: 0.91
    # the reference's actions of the golden points (disk-like: partly outside the training set)
    g = np.load(os.path.join(GOLDEN, "actions_cfg4.npz"))
    check_actions(af(g["points"]), g["act_finder"])
