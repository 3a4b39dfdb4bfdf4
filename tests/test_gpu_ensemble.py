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


def _ternary_fp32_members(seed=21):
    """A batched-run ensemble of the persistent kind: ternary FP32 members at
    256^2, 512^2 and 1024^2 with their own sigma_ij and noise."""
    rng = np.random.default_rng(seed)
    out = []
    for n, dt in ((1024, 3e-6), (256, 1e-4), (512, 2.5e-5), (256, 1e-4), (512, 2.5e-5), (256, 1e-4)):
        lx = 2 * math.pi
        p = dict(model=2, nx=n, ny=n, lx=lx, dt=dt, nu=0.01, precision=1, coef_mode=1, epsilon=2 * lx / n,
                 sigma12=0.2 + 0.05 * rng.uniform(), sigma13=0.3, sigma23=0.25 + 0.05 * rng.uniform(), xlambda=2.0)
        p["lambda"] = 0.005
        out.append((p, [1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n)), 1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n))]))
    return out


def test_persistent_step_matches_lone_contexts_and_the_graph(chns):
    """One persistent cooperative kernel per step (every member ternary FP32 at
    256..1024): each member bitwise equal to a lone context and to the same
    ensemble stepped by the graph of per-member branches."""
    members = _ternary_fp32_members()
    steps = 12
    states = {}
    for mode in (True, False):
        with chns.Ensemble([p for p, _ in members]) as ens:
            assert not ens.persistent  # the graph is the default
            ens.persistent = mode
            assert ens.persistent == mode
            for m, (_, ph) in zip(ens.members, members):
                m.set_phase_real(*ph)
            ens.step(steps - 4)
            ens.step(4)
            ens.synchronize()
            states[mode] = [m.get_state() for m in ens.members]
    for i, (p, ph) in enumerate(members):
        with chns.Context(p) as c:
            c.set_phase_real(*ph)
            c.step(steps)
            want = c.get_state()
        for a, b, w in zip(states[True][i], states[False][i], want):
            assert np.isfinite(a).all()
            assert np.array_equal(a, w), (i, p["nx"], "persistent vs lone")
            assert np.array_equal(b, w), (i, p["nx"], "graph vs lone")


def test_persistent_mode_needs_eligible_members(chns):
    members = _members()  # mixed models and precisions
    with chns.Ensemble([p for p, _ in members]) as ens:
        assert not ens.persistent
        with pytest.raises(chns.ChnsError) as ei:
            ens.persistent = True
        assert ei.value.status == -5
