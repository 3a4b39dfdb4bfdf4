"""Discrete adjoint of the binary ETD2RK step (chns_adjoint) against central
finite differences of the GPU forward step, and the FP32 adjoint against the
FP64 one.  The loss is the final-time free energy plus <|grad phi|^2>
(free_energy.c:3-157 with phi = 2c - 1), evaluated here with numpy on the final
state so the forward side of the check is independent of the adjoint code.
A torch.autograd.Function wraps the adjoint for the gradient check only.

Tolerance: directional derivatives match central differences (h = 1e-6,
relative) to 1e-6 relative in FP64."""
import math

import numpy as np
import pytest

from _golden import load_small

pytestmark = pytest.mark.gpu

STEPS, CKPT = 12, 5


def loss_numpy(p, c_hat, w=(1.0, 1.0, 1.0)):
    n = p["nx"]
    f = 2 * math.pi / p["lx"]
    kx = np.where(np.arange(n) <= n // 2, np.arange(n), np.arange(n) - n) * f
    ky = np.arange(n // 2 + 1) * f
    c = np.fft.irfft2(c_hat, s=(n, n))
    cx = np.fft.irfft2(1j * kx[:, None] * c_hat, s=(n, n))
    cy = np.fft.irfft2(1j * ky[None, :] * c_hat, s=(n, n))
    sg, ep = p["sigma"], p["epsilon"]
    eb = np.mean(12.0 * (sg / ep) * c * c * (1 - c) * (1 - c))
    eg = 0.75 * sg * ep * np.mean(cx * cx + cy * cy)
    gp = 4.0 * np.mean(cx * cx + cy * cy)
    return w[0] * eb + w[1] * eg + w[2] * gp


@pytest.fixture(scope="module")
def setup():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test needs a CUDA device")
    import chns_b200

    g = load_small("bin64")
    p = dict(g["params"], coef_mode=1, precision=0)
    return chns_b200, g, p


def forward_loss(C, p, state):
    with C.Context(p) as c:
        c.set_state(*state)
        c.step(STEPS)
        return loss_numpy(p, c.get_state()[1])


def rdot(a, b):
    return float(np.sum(a.real * b.real + a.imag * b.imag))


def test_adjoint_matches_finite_differences(setup):
    C, g, p = setup
    n = p["nx"]
    w0, c0 = g["init"]
    with C.Context(p) as c:
        c.set_state(w0, c0)
        J, gw, gc, gpar = c.adjoint(STEPS, CKPT)
    assert abs(J - forward_loss(C, p, [w0, c0])) <= 1e-12 * abs(J)
    rng = np.random.default_rng(3)
    for k in range(8):
        # smooth real perturbations of c and omega
        dc = np.fft.rfft2(rng.standard_normal((n, n)))
        dw = np.fft.rfft2(rng.standard_normal((n, n)))
        kk = np.sqrt(np.arange(n)[:, None] ** 2 + np.arange(n // 2 + 1)[None, :] ** 2)
        dc *= np.exp(-kk / 6.0) * np.abs(c0).max() / np.abs(dc).max()
        dw *= np.exp(-kk / 6.0) * max(np.abs(w0).max(), 1.0) / np.abs(dw).max()
        h = 1e-6
        fd = (forward_loss(C, p, [w0 + h * dw, c0 + h * dc]) - forward_loss(C, p, [w0 - h * dw, c0 - h * dc])) / (2 * h)
        ad = rdot(gw, dw) + rdot(gc, dc)
        assert abs(ad - fd) <= 1e-6 * abs(fd), (k, ad, fd)
    # parameters nu, lambda, sigma
    for i, key in enumerate(("nu", "lambda", "sigma")):
        h = 1e-6 * p[key]
        jp = forward_loss(C, dict(p, **{key: p[key] + h}), [w0, c0])
        jm = forward_loss(C, dict(p, **{key: p[key] - h}), [w0, c0])
        fd = (jp - jm) / (2 * h)
        assert abs(gpar[i] - fd) <= 1e-6 * abs(fd) + 1e-9 * abs(J) / p[key], (key, gpar[i], fd)


def test_fp32_adjoint_close_to_fp64(setup):
    C, g, p = setup
    w0, c0 = g["init"]
    out = []
    for prec in (0, 1):
        with C.Context(dict(p, precision=prec)) as c:
            c.set_state(w0, c0)
            out.append(c.adjoint(STEPS, CKPT))
    (J64, gw64, gc64, gp64), (J32, gw32, gc32, gp32) = out
    assert abs(J32 - J64) <= 1e-5 * abs(J64)
    assert np.linalg.norm(gc32 - gc64) <= 1e-3 * np.linalg.norm(gc64)
    assert np.allclose(gp32, gp64, rtol=1e-3, atol=0)


def test_autograd_function_wrapper(setup):
    """The gradient-check harness: a torch.autograd.Function whose backward is
    the hand-written adjoint."""
    import torch

    C, g, p = setup
    w0, c0 = g["init"]

    class FinalLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, c_re_im):
            ch = c_re_im.detach().cpu().numpy().view(np.complex128)[..., 0]
            with C.Context(p) as c:
                c.set_state(w0, ch)
                J, _, gc, _ = c.adjoint(STEPS, CKPT)
            ctx.save_for_backward(torch.from_numpy(gc.view(np.float64).reshape(c_re_im.shape)))
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gJ):
            (gc,) = ctx.saved_tensors
            return gJ * gc

    x = torch.from_numpy(np.ascontiguousarray(c0).view(np.float64).reshape(c0.shape + (2,)).copy())
    x.requires_grad_(True)
    J = FinalLoss.apply(x)
    (grad,) = torch.autograd.grad(J, x)
    n = p["nx"]
    d = np.fft.rfft2(np.random.default_rng(9).standard_normal((n, n)))
    d *= np.exp(-np.sqrt(np.arange(n)[:, None] ** 2 + np.arange(n // 2 + 1)[None, :] ** 2) / 6.0)
    d *= np.abs(c0).max() / np.abs(d).max()
    h = 1e-6
    fd = (forward_loss(C, p, [w0, c0 + h * d]) - forward_loss(C, p, [w0, c0 - h * d])) / (2 * h)
    ad = float(torch.sum(grad * torch.from_numpy(d.view(np.float64).reshape(d.shape + (2,)))))
    assert abs(ad - fd) <= 1e-6 * abs(fd)


def test_checkpoint_interval_does_not_change_gradients(setup):
    """Every checkpoint interval (one segment, several, one step per segment)
    reverses the same trajectory: results agree to round-off."""
    C, g, p = setup
    w0, c0 = g["init"]
    out = {}
    with C.Context(p) as c:
        c.set_state(w0, c0)
        for k in (1, 3, 5, 12, 40):
            out[k] = c.adjoint(STEPS, k)
        # the state is unchanged by the adjoint
        w1, c1 = c.get_state()
    assert np.array_equal(w1, w0) and np.array_equal(c1, c0)
    J0, gw0, gc0, gp0 = out[STEPS]
    for k, (J, gw, gc, gp) in out.items():
        assert abs(J - J0) <= 1e-14 * abs(J0), k
        assert np.linalg.norm(gc - gc0) <= 1e-13 * np.linalg.norm(gc0), k
        assert np.linalg.norm(gw - gw0) <= 1e-13 * max(np.linalg.norm(gw0), 1e-300), k
        assert np.allclose(gp, gp0, rtol=1e-12, atol=0), k


# ---------------------------------------------------------------------------
# ternary model: J = E_bulk + E_grad + <|grad c1|^2 + |grad c2|^2> (free_energy.c)
# ---------------------------------------------------------------------------
def gammas(p):
    s12, s13, s23 = p["sigma12"], p["sigma13"], p["sigma23"]
    return s12 - s23 + s13, s12 - s13 + s23, s23 - s12 + s13


def loss_numpy_ternary(p, c1_hat, c2_hat, w=(1.0, 1.0, 1.0)):
    n = p["nx"]
    f = 2 * math.pi / p["lx"]
    kx = np.where(np.arange(n) <= n // 2, np.arange(n), np.arange(n) - n) * f
    ky = np.arange(n // 2 + 1) * f
    g1, g2, g3 = gammas(p)
    eps = p["epsilon"]

    def real(h, mx=0, my=0):
        return np.fft.irfft2((1j * kx[:, None]) ** mx * (1j * ky[None, :]) ** my * h, s=(n, n))

    c1, c2 = real(c1_hat), real(c2_hat)
    c1x, c1y, c2x, c2y = real(c1_hat, 1), real(c1_hat, 0, 1), real(c2_hat, 1), real(c2_hat, 0, 1)
    c3 = 1 - c1 - c2
    eb = (6 / eps) * np.mean(g1 * c1 ** 2 * (1 - c1) ** 2 + g2 * c2 ** 2 * (1 - c2) ** 2
                             + g3 * c3 ** 2 * (c1 + c2) ** 2)
    eg = 0.375 * eps * np.mean(g1 * (c1x ** 2 + c1y ** 2) + g2 * (c2x ** 2 + c2y ** 2)
                               + g3 * ((c1x + c2x) ** 2 + (c1y + c2y) ** 2))
    gp = np.mean(c1x ** 2 + c1y ** 2 + c2x ** 2 + c2y ** 2)
    return w[0] * eb + w[1] * eg + w[2] * gp


@pytest.fixture(scope="module")
def tsetup():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test needs a CUDA device")
    import chns_b200

    g = load_small("ter64")
    p = dict(g["params"], coef_mode=1, precision=0)
    return chns_b200, g, p


def forward_loss_ternary(C, p, state):
    with C.Context(p) as c:
        c.set_state(*state)
        c.step(STEPS)
        st = c.get_state()
        return loss_numpy_ternary(p, st[1], st[2])


def test_ternary_adjoint_matches_finite_differences(tsetup):
    C, g, p = tsetup
    n = p["nx"]
    w0, a0, b0 = g["init"]
    with C.Context(p) as c:
        c.set_state(w0, a0, b0)
        J, gw, (g1, g2), gpar = c.adjoint(STEPS, CKPT)
        after = c.get_state()
    for x, y in zip(after, (w0, a0, b0)):
        assert np.array_equal(x, y)
    assert abs(J - forward_loss_ternary(C, p, [w0, a0, b0])) <= 1e-12 * abs(J)
    rng = np.random.default_rng(13)
    kk = np.sqrt(np.arange(n)[:, None] ** 2 + np.arange(n // 2 + 1)[None, :] ** 2)
    scale = max(np.abs(a0).ravel()[1:].max(), np.abs(b0).ravel()[1:].max())
    bad = []
    for k in range(8):
        ds = []
        for amp in (scale, scale, max(np.abs(w0).max(), 1.0)):
            d = np.fft.rfft2(rng.standard_normal((n, n))) * np.exp(-kk / 6.0)
            ds.append(d * amp / np.abs(d).max())
        d1, d2, dw = ds
        h = 1e-6
        jp = forward_loss_ternary(C, p, [w0 + h * dw, a0 + h * d1, b0 + h * d2])
        jm = forward_loss_ternary(C, p, [w0 - h * dw, a0 - h * d1, b0 - h * d2])
        fd = (jp - jm) / (2 * h)
        ad = rdot(gw, dw) + rdot(g1, d1) + rdot(g2, d2)
        # 1e-6 relative, above the difference quotient's rounding floor ~1e-15 |J| / (2h)
        bad.append((k, ad, fd)) if abs(ad - fd) > 1e-6 * abs(fd) + 1e-9 * abs(J) else None
    for i, key in enumerate(("nu", "lambda", "sigma12", "sigma13", "sigma23")):
        h = 1e-6 * p[key]
        jp = forward_loss_ternary(C, dict(p, **{key: p[key] + h}), [w0, a0, b0])
        jm = forward_loss_ternary(C, dict(p, **{key: p[key] - h}), [w0, a0, b0])
        fd = (jp - jm) / (2 * h)
        if abs(gpar[i] - fd) > 1e-6 * abs(fd) + 1e-9 * abs(J) / p[key]:
            bad.append((key, gpar[i], fd))
    assert not bad, (J, bad)


def test_ternary_fp32_adjoint_close_to_fp64(tsetup):
    C, g, p = tsetup
    out = []
    for prec in (0, 1):
        with C.Context(dict(p, precision=prec)) as c:
            c.set_state(*g["init"])
            out.append(c.adjoint(STEPS, CKPT))
    (J64, _, (a64, b64), gp64), (J32, _, (a32, b32), gp32) = out
    assert abs(J32 - J64) <= 1e-5 * abs(J64)
    assert np.linalg.norm(a32 - a64) <= 1e-3 * np.linalg.norm(a64)
    assert np.linalg.norm(b32 - b64) <= 1e-3 * np.linalg.norm(b64)
    assert np.allclose(gp32, gp64, rtol=1e-3, atol=1e-6 * np.abs(gp64).max())
