"""Discrete adjoint of the pure Navier-Stokes ETD2RK step (chns_adjoint on a
model-0 context) against central finite differences of the GPU forward step.
The loss is a_ke <|u|^2/2> + a_ens <w_t^2/2> of the truncated velocity and
vorticity at the final step (kinetic_energy.c:17-21,43-49,89), evaluated here with
numpy on the final state so the forward side of the check is independent of the
adjoint code.  Unforced and Kolmogorov-forced runs (the forcing is constant in
the state, so it only enters through the trajectory).

Tolerance: directional derivatives and dJ/dnu match central differences (h = 1e-6,
relative) to 1e-6 relative in FP64; the result does not depend on the checkpoint
interval; FP32 within 1e-3 of FP64."""
import math

import numpy as np
import pytest

from chns_b200 import fields

pytestmark = pytest.mark.gpu

STEPS, CKPT = 12, 5
N = 64


def loss_numpy(p, w_hat, lw=(1.0, 1.0)):
    n = p["nx"]
    f = 2 * math.pi / p["lx"]
    kx = np.where(np.arange(n) <= n // 2, np.arange(n), np.arange(n) - n) * f
    ky = np.arange(n // 2 + 1) * f
    ks = kx[:, None] ** 2 + ky[None, :] ** 2
    dax = (n / 4.0) * f
    keep = ks <= dax * dax                      # functions.c:47-84
    psi = np.where(ks > 1e-12, w_hat / np.where(ks > 1e-12, ks, 1.0), 0.0)
    u = np.fft.irfft2(np.where(keep, 1j * ky[None, :] * psi, 0.0), s=(n, n))
    v = np.fft.irfft2(np.where(keep, -1j * kx[:, None] * psi, 0.0), s=(n, n))
    wt = np.fft.irfft2(np.where(keep, w_hat, 0.0), s=(n, n))
    return lw[0] * np.mean(0.5 * (u * u + v * v)) + lw[1] * np.mean(0.5 * wt * wt)


def rdot(a, b):
    return float(np.sum(a.real * b.real + a.imag * b.imag))


@pytest.fixture(scope="module")
def chns():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test needs a CUDA device")
    import chns_b200

    chns_b200.load_library()
    return chns_b200


def _params(forced, prec=0):
    p = dict(model=0, nx=N, ny=N, lx=2 * math.pi, ly=2 * math.pi, dt=2e-3, nu=0.01, coef_mode=1, precision=prec)
    if forced:
        p.update(force_amp=1.0, force_k=4.0)
    return p


def forward_loss(C, p, w, lw=(1.0, 1.0)):
    with C.Context(p) as c:
        c.set_state(w)
        c.step(STEPS)
        return loss_numpy(p, c.get_state()[0], lw)


@pytest.mark.parametrize("forced", [False, True])
def test_ns_adjoint_matches_finite_differences(chns, forced):
    p = _params(forced)
    w0 = fields.random_vorticity_hat(N, 11, kmax=8.0, rms=1.0, lx=p["lx"])
    lw = (1.0, 0.3)
    with chns.Context(p) as c:
        c.set_state(w0)
        J, gw, gc, gpar = c.adjoint(STEPS, CKPT, loss_w=(lw[0], lw[1], 0.0))
        assert gc is None
        assert np.array_equal(c.get_state()[0], w0)  # the state is unchanged
    assert abs(J - forward_loss(chns, p, w0, lw)) <= 1e-12 * abs(J)
    rng = np.random.default_rng(5)
    kk = np.sqrt(np.arange(N)[:, None] ** 2 + np.arange(N // 2 + 1)[None, :] ** 2)
    for k in range(8):
        dw = np.fft.rfft2(rng.standard_normal((N, N)))
        dw *= np.exp(-kk / 6.0) * np.abs(w0).max() / np.abs(dw).max()
        h = 1e-6
        fd = (forward_loss(chns, p, w0 + h * dw, lw) - forward_loss(chns, p, w0 - h * dw, lw)) / (2 * h)
        ad = rdot(gw, dw)
        assert abs(ad - fd) <= 1e-6 * abs(fd), (k, ad, fd)
    h = 1e-6 * p["nu"]
    fd = (forward_loss(chns, dict(p, nu=p["nu"] + h), w0, lw) - forward_loss(chns, dict(p, nu=p["nu"] - h), w0, lw)) / (2 * h)
    assert abs(gpar[0] - fd) <= 1e-6 * abs(fd), (gpar[0], fd)
    assert gpar[1] == 0.0 and gpar[2] == 0.0


def test_ns_adjoint_independent_of_checkpoints_and_fp32_close(chns):
    p = _params(True)
    w0 = fields.random_vorticity_hat(N, 12, kmax=8.0, rms=1.0, lx=p["lx"])
    out = []
    for ck in (1, 3, 12, 40):
        with chns.Context(p) as c:
            c.set_state(w0)
            out.append(c.adjoint(STEPS, ck))
    for J, gw, _, gp in out[1:]:
        assert abs(J - out[0][0]) <= 1e-13 * abs(out[0][0])
        assert np.linalg.norm(gw - out[0][1]) <= 1e-12 * np.linalg.norm(out[0][1])
        assert abs(gp[0] - out[0][3][0]) <= 1e-11 * abs(out[0][3][0])
    with chns.Context(dict(p, precision=1)) as c:
        c.set_state(w0)
        J32, gw32, _, gp32 = c.adjoint(STEPS, CKPT)
    assert abs(J32 - out[0][0]) <= 1e-5 * abs(out[0][0])
    assert np.linalg.norm(gw32 - out[0][1]) <= 1e-3 * np.linalg.norm(out[0][1])
    assert abs(gp32[0] - out[0][3][0]) <= 1e-3 * abs(out[0][3][0])
