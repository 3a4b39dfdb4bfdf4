"""GPU parity tests: the sm_100a path through the C ABI against the oracle
(the reference's own code run here: golden fixtures, and the C restatement).

Tolerances: FP64 relative L2 <= 1e-11 after 20 steps on small grids and
<= 1e-10 after 1000 / 2000 steps on the binary 256^2 and ternary 512^2 runs (the only
differences are FFT round-off, ~1e-16 per transform); FP32 <= 1e-5.
"""
import math

import numpy as np
import pytest

import make_golden as MG
from _golden import SMALL_CONFIGS, load_full, load_small, rel_l2

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


@pytest.mark.parametrize("n", [32, 64, 128, 256, 512, 1024, 2048, 4096])
@pytest.mark.parametrize("prec", [0, 1])
def test_fft_vs_numpy(chns, n, prec):
    p = dict(model=0, nx=n, ny=n, lx=2 * math.pi, dt=1e-3, nu=0.01, precision=prec)
    with _ctx(chns, p) as c:
        rng = np.random.default_rng(n)
        x = rng.standard_normal((n, n))
        X = c.dfft(x)
        ref = np.fft.rfft2(x)
        tol = 1e-13 if prec == 0 else 2e-6
        assert rel_l2(X, ref) <= tol
        y = c.ifft(ref)
        assert rel_l2(y, x) <= tol
        # c2r of a non-Hermitian half spectrum: Im of the ky = 0, n/2 bins ignored
        Z = rng.standard_normal(X.shape) + 1j * rng.standard_normal(X.shape)
        assert rel_l2(c.ifft(Z), np.fft.irfft2(Z, s=(n, n))) <= tol


@pytest.mark.parametrize("n", [256, 1024, 4096])
@pytest.mark.parametrize("prec", [0, 1])
def test_fft_vs_cufft(chns, n, prec):
    """Cross-check of the own transforms against cuFFT (torch.fft on the same GPU)
    in the same precision: FP64 <= 1e-13, FP32 <= 2e-6 relative L2."""
    import torch

    p = dict(model=0, nx=n, ny=n, lx=2 * math.pi, dt=1e-3, nu=0.01, precision=prec)
    dt = torch.float64 if prec == 0 else torch.float32
    with _ctx(chns, p) as c:
        rng = np.random.default_rng(n + 7)
        x = rng.standard_normal((n, n))
        ref = torch.fft.rfft2(torch.from_numpy(x).to("cuda", dt)).cpu().numpy().astype(np.complex128)
        tol = 1e-13 if prec == 0 else 2e-6
        assert rel_l2(c.dfft(x), ref) <= tol
        back = torch.fft.irfft2(torch.from_numpy(ref).to("cuda"), s=(n, n)).cpu().numpy()
        assert rel_l2(c.ifft(ref), back) <= tol


@pytest.mark.parametrize("model,n", [(1, 32), (1, 64), (1, 256), (1, 512), (1, 2048), (1, 4096), (0, 128),
                                     (0, 1024), (2, 128), (2, 1024)])
def test_row_tiles_by_tma(chns, model, n):
    """The row kernels load their tiles with TMA (tensor maps encoded at context
    creation, FP32 and FP64); no tile wait runs out over a few steps (chns_check
    would return CHNS_ERR_TIMEOUT), and the FP32 state stays within 1e-5 of the FP64
    one."""
    rng = np.random.default_rng(n)
    lx = 2 * math.pi
    p = dict(model=model, nx=n, ny=n, lx=lx, dt=1e-6, nu=0.01, sigma=0.2, epsilon=2 * lx / n, coef_mode=1,
             sigma12=0.2, sigma13=0.3, sigma23=0.25)
    p["lambda"] = 0.005
    ph = [0.5 + 0.05 * rng.uniform(-1, 1, (n, n)) for _ in range(model)]
    w = np.zeros((n, n // 2 + 1), np.complex128)
    w[1, 2], w[3, 1] = 0.3 * n * n, 0.2 * n * n  # a few vorticity modes (ky > 0: no Hermitian pairing)
    res = []
    for prec in (0, 1):
        with _ctx(chns, p, precision=prec) as c:
            assert c.tma_tiles()
            if model:
                c.set_phase_real(*ph)
            st = c.get_state()
            st[0] = w
            c.set_state(*st)
            c.step(3)
            c.check()
            res.append(c.get_state())
    for a, b in zip(res[1], res[0]):
        assert rel_l2(a, b) <= 1e-5


@pytest.mark.parametrize("name", SMALL_CONFIGS)
def test_rhs_matches_reference(chns, name):
    g = load_small(name)
    with _ctx(chns, g["params"]) as c:
        c.set_state(*g["init"])
        for k, (a, b) in enumerate(zip(c.rhs(), g["rhs"])):
            assert rel_l2(a, b) <= 1e-12, (name, k, rel_l2(a, b))
        # the state is unchanged by rhs()
        for a, b in zip(c.get_state(), g["init"]):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("name", SMALL_CONFIGS)
def test_steps_match_reference(chns, name):
    g = load_small(name)
    with _ctx(chns, g["params"]) as c:
        c.set_state(*g["init"])
        c.step(g["steps"])
        for k, (a, b) in enumerate(zip(c.get_state(), g["final"])):
            assert rel_l2(a, b) <= 1e-11, (name, k, rel_l2(a, b))


@pytest.mark.parametrize("name", ["bin32", "ter32", "bindef64", "terdef64", "binsf64", "tersf64", "binsfdef64"])
def test_diagnostics_match_reference(chns, name):
    g = load_small(name)
    with _ctx(chns, g["params"]) as c:
        c.set_state(*g["init"])
        fe, ke, rc = c.diagnostics()
        assert rc == 0
        assert np.allclose(fe, g["fe0"], rtol=1e-11, atol=1e-12)
        nk = len(g["ke0"])
        assert np.allclose(ke[:nk], g["ke0"], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("name", ["bin64", "ter64", "binsf64", "tersf64"])
def test_phase_init_matches_reference(chns, name):
    """init.c INIT_READ_DATA path: dfft + truncation of the real phase fields."""
    g = load_small(name)
    p = g["params"]
    p1, p2, _ = MG.initial_state(p["model"], p["nx"], p["lx"], 1 if p["model"] == 1 else 2, None, 0, 0)
    with _ctx(chns, p) as c:
        c.set_phase_real(p1, p2)
        st = c.get_state()
        for k in range(1, p["model"] + 1):
            assert rel_l2(st[k], g["init"][k]) <= 1e-14
        assert np.abs(st[0]).max() == 0.0


@pytest.mark.parametrize("name,seed", [("bin256", 100), ("ter512", 101)])
def test_baseline_configs_match_reference(chns, name, seed):
    """The binary 256^2 (1000 steps) and ternary 512^2 (2000 steps, dt = 5e-5)
    spinodal runs against the reference's run: every field (omega and each c_i)
    within 1e-10 relative L2 of the reference's final state, its fingerprint (low
    modes, random projections, norm) too, mean concentration conserved to
    round-off."""
    g = load_full(name)
    p = g["params"]
    p1, p2, w = MG.initial_state(p["model"], p["nx"], p["lx"], seed, None, 0, 0)
    with _ctx(chns, p) as c:
        c.set_phase_real(p1, p2)
        st0 = c.get_state()
        c.step(g["steps"])
        st = c.get_state()
    for k, a in enumerate(st):
        ref_field = g[f"final{k}"]
        if k == 0 and not np.any(ref_field):
            assert not np.any(a), (name, "omega stays zero")
        else:
            err = rel_l2(a, ref_field)
            assert err <= 1e-10, (name, k, err)
        fp = MG.fingerprint(a)
        ref = {key: g[f"final{k}_{key}"] for key in ("low", "proj", "norm")}
        err = MG.fingerprint_rel_err(ref, fp)
        assert err <= 1e-10, (name, k, err)
    for k in range(1, p["model"] + 1):
        assert abs(st[k][0, 0] - st0[k][0, 0]) <= 1e-12 * abs(st0[k][0, 0])


@pytest.mark.parametrize("name", ["bin64", "ter64"])
def test_fp32_close_to_fp64(chns, name):
    g = load_small(name)
    p = g["params"]
    with _ctx(chns, p) as a, _ctx(chns, p, precision=1, coef_mode=1) as b:
        a.set_state(*g["init"])
        b.set_state(*g["init"])
        a.step(20)
        b.step(20)
        for x, y in zip(b.get_state(), a.get_state()):
            assert rel_l2(x, y) <= 1e-5
        # k = 0 modes are carried in double in FP32 contexts
        for x, y in zip(b.get_state()[1:], a.get_state()[1:]):
            assert abs(x[0, 0] - y[0, 0]) <= 1e-9 * abs(y[0, 0])


def test_kolmogorov_forcing_matches_oracle(chns):
    import oracle as O

    n = 64
    p = dict(model=1, nx=n, ny=n, lx=2 * math.pi, ly=2 * math.pi, dt=2e-4, nu=1e-3, sigma=0.1,
             epsilon=2.0 * (2 * math.pi / n), coef_mode=0, force_amp=1.0, force_k=4.0)
    p["lambda"] = 1e-3
    o = O.Oracle(p)
    c1 = MG.fields.drops_binary(n, 7, ndrops=4, radius=0.6)
    w = MG.fields.random_vorticity_hat(n, 8, kmax=4.0, rms=0.1)
    MG.apply_initial(o, 1, c1, None, w)
    st0 = o.get_state()
    o.step(10)
    with _ctx(chns, p) as c:
        c.set_state(*st0)
        c.step(10)
        for a, b in zip(c.get_state(), o.get_state()):
            assert rel_l2(a, b) <= 1e-11


@pytest.mark.parametrize("case", MG.BIG, ids=[c[0] for c in MG.BIG])
def test_large_grids_match_reference(chns, case):
    """The 4096^2 binary and 1024^2 ternary kernels against the reference's own
    steps (compiled here) from spinodal noise plus random low-k vorticity:
    fingerprint within 1e-11 after 2-3 steps."""
    name, steps, ps, ws, kmax, rms = case
    g = load_full(name)
    p = g["params"]
    assert g["steps"] == steps
    p1, p2, w = MG.initial_state(p["model"], p["nx"], p["lx"], ps, ws, kmax, rms)
    with _ctx(chns, p) as c:
        MG.apply_initial(c, p["model"], p1, p2, w)
        c.step(steps)
        st = c.get_state()
    for k, a in enumerate(st):
        fp = MG.fingerprint(a)
        ref = {key: g[f"final{k}_{key}"] for key in ("low", "proj", "norm")}
        err = MG.fingerprint_rel_err(ref, fp)
        assert err <= 1e-11, (name, k, err)
