"""CHNS_FP32_STATE64: FP32 right-hand side, the state carried as a float pair
hi + lo (48 significant bits) and the ETD update done in float-float arithmetic.

The state given to chns_set_state comes back to 2^-48 per element inside the
truncation disc (the modes that reach a right-hand side) and 2^-24 outside; the low part
stays consistent with the float part the right-hand side reads (initial
conditions, chns_rhs, ensembles, checkpoints); and the trajectory is much closer
to the FP64 step than the plain FP32 one, because the rounding of every small
increment into a float state is what the spinodal modes amplify.  Tolerances:
<= 1e-6 relative L2 against FP64 after 20 steps of the small golden cases; on the
forced drop run the error must be at most a tenth of the FP32 run's.
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


def _ctx(chns, p, **kw):
    q = dict(p)
    q.update(kw)
    return chns.Context(q)


@pytest.mark.parametrize("name", ["bin64", "ter64", "ns32"])
def test_state_round_trip(chns, name):
    g = load_small(name)
    with _ctx(chns, g["params"], precision=chns.FP32_STATE64) as c:
        c.set_state(*g["init"])
        st = c.get_state()
    n = g["params"]["nx"]
    kx = np.where(np.arange(n) <= n // 2, np.arange(n), np.arange(n) - n)[:, None]
    ky = np.arange(n // 2 + 1)[None, :]
    disc = kx ** 2 + ky ** 2 <= (n / 4) ** 2  # functions.c:56-59 with lx = 2 pi
    for a, b in zip(st, g["init"]):
        err = np.abs(a - b)
        assert np.all(err[disc] <= 2.0 ** -47 * np.abs(b[disc]))
        assert np.all(err <= 2.0 ** -23 * np.abs(b))
        assert a[0, 0] == b[0, 0]  # the k = 0 mode is kept in double


@pytest.mark.parametrize("name", ["bin64", "ter64"])
def test_closer_to_fp64_than_fp32(chns, name):
    g = load_small(name)
    p = g["params"]
    res = {}
    for prec in (chns.FP64, chns.FP32, chns.FP32_STATE64):
        with _ctx(chns, p, precision=prec, coef_mode=1) as c:
            c.set_state(*g["init"])
            c.step(20)
            res[prec] = c.get_state()
    for k in range(len(res[chns.FP64])):
        e32 = rel_l2(res[chns.FP32][k], res[chns.FP64][k])
        e64 = rel_l2(res[chns.FP32_STATE64][k], res[chns.FP64][k])
        assert e64 <= 1e-6, (name, k, e64)
        assert e64 <= e32, (name, k, e64, e32)


def test_forced_drops_error_tenfold_below_fp32(chns):
    """The forced drop workload at 512^2 (dt = 1e-4, 300 steps): the FP32 state's
    error comes from rounding small increments (measured in a cuFFT emulation of
    this run: w 2.5e-5 against 3.5e-7, c 6.5e-6 against 3.4e-8)."""
    from chns_b200 import configs

    n = 512
    p, c0, w0 = configs.binary_kolmogorov(n, dt=1e-4)
    with _ctx(chns, p, precision=chns.FP64) as c:
        c.set_phase_real(c0)
        st0 = c.get_state()
    st0[0] = w0
    res = {}
    for prec in (chns.FP64, chns.FP32, chns.FP32_STATE64):
        with _ctx(chns, p, precision=prec) as c:
            c.set_state(*st0)
            c.step(300)
            c.check()
            res[prec] = c.get_state()
    for k in range(2):
        e32 = rel_l2(res[chns.FP32][k], res[chns.FP64][k])
        e64 = rel_l2(res[chns.FP32_STATE64][k], res[chns.FP64][k])
        assert e64 <= 0.1 * e32, (k, e64, e32)


@pytest.mark.parametrize("model", [1, 2])
def test_phase_initialisation_matches_fp32(chns, model):
    """Initial conditions written as float (set_phase_real, init_vorticity) reach
    the double state: get_state equals the FP32 context's (k = 0 from its double
    mode)."""
    n = 64
    rng = np.random.default_rng(5)
    lx = 2 * math.pi
    p = dict(model=model, nx=n, ny=n, lx=lx, dt=1e-4, nu=0.01, epsilon=2 * lx / n, sigma=0.2, sigma12=0.2,
             sigma13=0.3, sigma23=0.25)
    p["lambda"] = 0.005
    ph = [0.5 + 0.05 * rng.uniform(-1, 1, (n, n)) for _ in range(model)]
    got = {}
    for prec in (chns.FP32, chns.FP32_STATE64):
        with _ctx(chns, p, precision=prec) as c:
            c.set_phase_real(*ph)
            c.init_vorticity(chns.INIT_W_TAYLOR_GREEN, 0.5)
            got[prec] = c.get_state()
    for a, b in zip(got[chns.FP32], got[chns.FP32_STATE64]):
        assert np.array_equal(a, b)


def test_rhs_leaves_state_unchanged(chns):
    g = load_small("bin64")
    with _ctx(chns, g["params"], precision=chns.FP32_STATE64) as c:
        c.set_state(*g["init"])
        c.step(3)
        before = c.get_state()
        c.rhs()
        after = c.get_state()
        c.step(2)
        again = c.get_state()
    with _ctx(chns, g["params"], precision=chns.FP32_STATE64) as c:
        c.set_state(*g["init"])
        c.step(5)
        ref = c.get_state()
    for a, b in zip(before, after):
        assert np.array_equal(a, b)
    for a, b in zip(again, ref):
        assert np.array_equal(a, b)


def test_ensemble_member_matches_lone_context(chns):
    g = load_small("ter64")
    b = load_small("bin64")
    ps = [dict(g["params"], precision=chns.FP32_STATE64), dict(b["params"], precision=chns.FP32_STATE64),
          dict(b["params"], precision=chns.FP32)]
    inits = [g["init"], b["init"], b["init"]]
    with chns.Ensemble(ps) as ens:
        for m, st in zip(ens.members, inits):
            m.set_state(*st)
        ens.step(12)
        got = [m.get_state() for m in ens.members]
    for p, st, gs in zip(ps, inits, got):
        with chns.Context(p) as c:
            c.set_state(*st)
            c.step(12)
            for x, y in zip(gs, c.get_state()):
                assert np.array_equal(x, y)


def test_adjoint_rejects_double_state(chns):
    g = load_small("bin64")
    with _ctx(chns, g["params"], precision=chns.FP32_STATE64) as c:
        c.set_state(*g["init"])
        with pytest.raises(chns.ChnsError) as ei:
            c.adjoint(2, 1)
        assert ei.value.status == -5


def test_checkpoint_keeps_double_state(chns, tmp_path):
    g = load_small("bin64")
    path = str(tmp_path / "s64.ckpt")
    with _ctx(chns, g["params"], precision=chns.FP32_STATE64) as c:
        c.set_state(*g["init"])
        c.step(4)
        c.save(path)
        want = c.get_state()
    with _ctx(chns, g["params"], precision=chns.FP32_STATE64) as c:
        c.load(path)
        for a, b in zip(c.get_state(), want):
            assert rel_l2(a, b) <= 1e-15


def test_forced_drops_4096_within_1e5_of_fp64(chns):
    """The benchmark's 4096^2 forced drop workload (dt = 2e-6, so t = 0.002), the
    full 1000 steps: the float-pair state within 1e-5 relative L2 of the FP64
    step in omega and in c, the plain FP32 state further away."""
    from chns_b200 import configs

    n = 4096
    p, c0, w0 = configs.binary_kolmogorov(n, dt=2e-6)
    p["coef_mode"] = 1
    with _ctx(chns, p, precision=chns.FP64) as c:
        c.set_phase_real(c0)
        st0 = c.get_state()
    st0[0] = w0
    res = {}
    for prec in (chns.FP64, chns.FP32, chns.FP32_STATE64):
        with _ctx(chns, p, precision=prec) as c:
            c.set_state(*st0)
            c.step(1000)
            c.check()
            res[prec] = c.get_state()
    for k in range(2):
        e64 = rel_l2(res[chns.FP32_STATE64][k], res[chns.FP64][k])
        e32 = rel_l2(res[chns.FP32][k], res[chns.FP64][k])
        assert e64 <= 1e-5, (k, e64)
        assert e64 <= e32, (k, e64, e32)


def test_ternary_spinodal_4096_fp32_within_1e5_of_fp64(chns):
    """The ternary model at 4096^2 from spinodal noise (c_i = 1/3 + U[-0.02, 0.02],
    sigma_ij = 0.2/0.3/0.25, dt = 5e-8, 100 steps, the bench's ternary leg): both
    FP32 modes within 1e-5 relative L2 of the FP64 step in omega, c1 and c2.  The
    FP32 phase fields are transformed without their means (kept in double), at the
    initial transform and in the step's chemical potential; before, the means'
    rounding put the FP32 fields 2.5e-5 to 4.7e-5 away."""
    from chns_b200 import configs

    n = 4096
    p = configs.ternary(n, 5e-8, 0.01, 0.005, 0.2, 0.3, 0.25, coef_mode=1)
    rng = np.random.default_rng(7)
    ph = (1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n)), 1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n)))
    res = {}
    for prec in (chns.FP64, chns.FP32, chns.FP32_STATE64):
        with _ctx(chns, p, precision=prec) as c:
            c.set_phase_real(*ph)
            c.step(100)
            c.check()
            res[prec] = c.get_state()
    for prec in (chns.FP32, chns.FP32_STATE64):
        for k in range(3):
            e = rel_l2(res[prec][k], res[chns.FP64][k])
            assert e <= 1e-5, (prec, k, e)
