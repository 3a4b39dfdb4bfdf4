"""The discrete adjoint at the size of the benchmark's gradient check: binary
CHNS 512^2, 200 ETD2RK steps, checkpoints every 20 steps, FP64 (dt = 1e-4: the
spinodal setting of configs.binary_adjoint).  The loss is the final-time free
energy plus <|grad phi|^2> (free_energy.c:3-157, phi = 2c - 1), as chns_adjoint
returns it.

Directional derivatives along 8 seeded smooth directions of the initial
(omega_hat, c_hat) and the nu, M and sigma derivatives are compared with central
differences of the GPU forward map, at 1e-6 relative in every direction.  The
difference quotient is the fourth-order central one,
(8 (J(h) - J(-h)) - (J(2h) - J(-2h))) / (12 h), with the direction scaled to the
state's largest mode.  Its error is truncation, O(h^4), plus the rounding of J
(~1.6e3, carried through a spinodal trajectory) over h |dJ|; the directional
derivatives differ by 30x between directions, so no one h suits all of them.  For
each direction the quotient is taken at the step of a fixed ladder where it agrees
best with the quotient at the next step (the step-halving error estimate of
Richardson extrapolation, computed from J alone, never from the adjoint).  A
sweep of h on a B200 put the quotient's error below 1e-6 for every direction at
h = 1e-4 .. 1e-3; the second-order quotient at h = 1e-6 is limited by the rounding
of J to about 1e-6 itself."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, STEPS, CKPT = 512, 200, 20
H_LADDER = (3e-5, 1e-4, 3e-4, 1e-3)      # directions of the state (scaled to its largest mode)
H_LADDER_PARAM = (1e-6, 1e-5, 1e-4)      # relative steps of nu, M, sigma
TOL = 1e-6


@pytest.fixture(scope="module")
def case():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test needs a CUDA device")
    import chns_b200
    from chns_b200 import configs

    p, c_real = configs.binary_adjoint(N, chns_b200.FP64, 1e-4)
    with chns_b200.Context(p) as c:
        c.set_phase_real(c_real)
        st0 = c.get_state()
        adj = c.adjoint(STEPS, CKPT)
    return chns_b200, p, st0, adj


def _loss(C, p, w, c_hat):
    with C.Context(p) as c:
        c.set_state(w, c_hat)
        return c.adjoint(STEPS, CKPT)[0]


def _fd4(f, h):
    return (8.0 * (f(h) - f(-h)) - (f(2 * h) - f(-2 * h))) / (12.0 * h)


def _fd4_selected(f, ladder):
    """The fourth-order quotient at the ladder step whose value agrees best with
    the next step's (relative difference); returns (quotient, step, that difference)."""
    q = [_fd4(f, h) for h in ladder]
    k = min(range(len(q) - 1), key=lambda i: abs(q[i] - q[i + 1]) / abs(q[i + 1]))
    return q[k], ladder[k], abs(q[k] - q[k + 1]) / abs(q[k + 1])


def _rdot(a, b):
    return float(np.sum(a.real * b.real + a.imag * b.imag))


def test_adjoint_512_matches_central_differences_along_8_directions(case):
    C, p, (w0, c0), (J, gw, gc, gp) = case
    mx = np.minimum(np.arange(N), N - np.arange(N))
    kk = np.sqrt(mx[:, None] ** 2 + np.arange(N // 2 + 1)[None, :] ** 2)
    cmax = np.abs(c0).ravel()[1:].max()
    errs = []
    for k in range(8):
        rng = np.random.default_rng(500 + k)
        dc = np.fft.rfft2(rng.standard_normal((N, N))) * np.exp(-kk / 8.0)
        dc *= cmax / np.abs(dc).max()
        dc[0, 0] = 0.0
        # half the directions also move omega (omega_0 = 0: scaled like c)
        dw = np.zeros_like(dc)
        if k % 2:
            dw = np.fft.rfft2(rng.standard_normal((N, N))) * np.exp(-kk / 8.0)
            dw *= cmax / np.abs(dw).max()
            dw[0, 0] = 0.0
        fd, h, spread = _fd4_selected(lambda h: _loss(C, p, w0 + h * dw, c0 + h * dc), H_LADDER)
        ad = _rdot(gw, dw) + _rdot(gc, dc)
        errs.append(abs(ad - fd) / abs(fd))
        print(f"direction {k}: dJ {ad:+.6e}  h {h:g}  quotient spread {spread:.1e}  rel err {errs[-1]:.2e}")
    assert max(errs) <= TOL, errs


def test_adjoint_512_parameter_derivatives(case):
    C, p, (w0, c0), (J, gw, gc, gp) = case
    errs = {}
    for i, key in enumerate(("nu", "lambda", "sigma")):
        base = p[key]
        fd, h, spread = _fd4_selected(lambda h: _loss(C, dict(p, **{key: base * (1.0 + h)}), w0, c0),
                                      H_LADDER_PARAM)
        fd /= base
        errs[key] = abs(gp[i] - fd) / abs(fd)
        print(f"{key}: dJ {gp[i]:+.6e}  h {h:g}  quotient spread {spread:.1e}  rel err {errs[key]:.2e}")
    assert max(errs.values()) <= TOL, errs
