"""Ensembles (chns_ensemble_*): members with their own models, sizes, precisions,
parameters and seeds advanced by one graph launch per step.  Every member must
evolve exactly as a lone context with the same parameters (bitwise: the same
kernels run on the same data), and a member set up like a golden case must
match the reference's golden vectors (FP64 relative L2 <= 1e-11 after its steps).
"""
import math

import numpy as np
import pytest

from _golden import load_small, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def chns():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import chns_b200

    chns_b200.load_library()
    return chns_b200


def _members():
    """(params, initial phase fields) of a mixed ensemble."""
    out = []
    rng = np.random.default_rng(11)
    for k, (model, n, prec) in enumerate([(2, 32, 0), (2, 32, 1), (1, 64, 0), (1, 64, 1), (2, 64, 1), (0, 32, 0),
                                          (2, 128, 1), (1, 128, 0)]):
        lx = 2 * math.pi
        p = dict(model=model, nx=n, ny=n, lx=lx, dt=2e-4, nu=0.01, precision=prec, coef_mode=k % 2,
                 epsilon=2 * lx / n, sigma=0.2, sigma12=rng.uniform(0.15, 0.35), sigma13=rng.uniform(0.15, 0.35),
                 sigma23=rng.uniform(0.15, 0.35))
        p["lambda"] = 0.005
        if model == 2:
            ph = [1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n)), 1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n))]
        elif model == 1:
            ph = [0.5 + 0.05 * rng.uniform(-1, 1, (n, n))]
        else:
            ph = []
            p["force_amp"], p["force_k"] = 1.0, 2.0
        out.append((p, ph))
    return out


def test_members_match_lone_contexts(chns):
    members = _members()
    steps = 15
    with chns.Ensemble([p for p, _ in members]) as ens:
        assert len(ens) == len(members)
        for m, (p, ph) in zip(ens.members, members):
            if ph:
                m.set_phase_real(*ph)
        ens.step(steps - 5)
        ens.step(5)
        ens.synchronize()
        got = [m.get_state() for m in ens.members]
    for (p, ph), g in zip(members, got):
        with chns.Context(p) as c:
            if ph:
                c.set_phase_real(*ph)
            c.step(steps)
            want = c.get_state()
        for a, b in zip(g, want):
            assert np.array_equal(a, b), (p["model"], p["nx"], p["precision"])
            assert np.all(np.isfinite(a))


def test_member_matches_golden(chns):
    g = load_small("bin32")
    t = load_small("ter32")
    with chns.Ensemble([g["params"], t["params"], g["params"]]) as ens:
        ens.members[0].set_state(*g["init"])
        ens.members[1].set_state(*t["init"])
        ens.members[2].set_state(*g["init"])
        assert g["steps"] == t["steps"]
        ens.step(g["steps"])
        for i, ref in ((0, g), (1, t), (2, g)):
            st = ens.members[i].get_state()
            for a, b in zip(st, ref["final"]):
                assert rel_l2(a, b) <= 1e-11


def test_member_calls_between_ensemble_steps(chns):
    """Per-member work on member streams and ensemble steps stay ordered."""
    g = load_small("bin32")
    with chns.Ensemble([g["params"]] * 4) as ens:
        for m in ens.members:
            m.set_state(*g["init"])
        ens.step(3)
        ens.members[2].set_state(*g["init"])  # restart one member
        ens.step(g["steps"] - 3)
        ens.members[2].step(3)
        fe = [m.diagnostics()[0] for m in ens.members]
        final = [m.get_state() for m in ens.members]
    for i in (0, 1, 3):
        for a, b in zip(final[i], g["final"]):
            assert rel_l2(a, b) <= 1e-11
    for a, b in zip(final[2], g["final"]):
        assert rel_l2(a, b) <= 1e-11
    assert all(np.all(np.isfinite(f)) for f in fe)
