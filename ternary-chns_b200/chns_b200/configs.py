"""Named run configurations: the reference's compile-time settings (global.h,
macro.h) as run-time parameter dicts for Context / Ensemble, with their seeded
initial states (chns_b200.fields).  Each function documents where it departs from
the configuration it is named after and why.

  binary_spinodal      binary, 256^2, L = 2 pi, dt = 1e-3, nu = 0.01, M = 0.005,
                       eps = 2 dx, sigma = 0.2; spinodal noise (1000 steps)
  ternary_spinodal     ternary, 512^2, sigma_12/13/23 = 0.2/0.3/0.25; dt = 5e-5
                       (5e-4 diverges in the reference's own scheme)
  binary_kolmogorov    binary, 4096^2, Kolmogorov forcing F0 sin(4y), 64 drops,
                       nu = M = 1e-3, sigma = 0.1, eps = 2 dx; dt = 2e-6 (2e-4
                       diverges at this resolution); FP32 by default
  ternary_ensemble     64 ternary runs (32 x 256^2, 24 x 512^2, 8 x 1024^2) with
                       sigma_ij ~ U[0.15, 0.35] (every gamma_i >= 0.1), FP32
  binary_adjoint       the binary spinodal setting at 512^2 for the adjoint,
                       dt = 1e-4 (1e-3 diverges at 512^2 with eps = 2 dx)
"""
from __future__ import annotations

import math

import numpy as np

from . import fields

TWO_PI = 2.0 * math.pi


def binary(n: int, dt: float, nu: float, mobility: float, sigma: float, precision: int = 0,
           coef_mode: int = 1, lx: float = TWO_PI, eps_cells: float = 2.0, force_amp: float = 0.0,
           force_k: float = 0.0) -> dict:
    p = dict(model=1, precision=precision, nx=n, ny=n, lx=lx, ly=lx, dt=dt, nu=nu, sigma=sigma,
             epsilon=eps_cells * (lx / n), coef_mode=coef_mode, force_amp=force_amp, force_k=force_k)
    p["lambda"] = mobility
    return p


def ternary(n: int, dt: float, nu: float, mobility: float, s12: float, s13: float, s23: float,
            precision: int = 0, coef_mode: int = 1, lx: float = TWO_PI, eps_cells: float = 2.0,
            xlambda: float = 2.0) -> dict:
    p = dict(model=2, precision=precision, nx=n, ny=n, lx=lx, ly=lx, dt=dt, nu=nu, epsilon=eps_cells * (lx / n),
             sigma12=s12, sigma13=s13, sigma23=s23, xlambda=xlambda, coef_mode=coef_mode)
    p["lambda"] = mobility
    return p


def binary_spinodal(n: int = 256, precision: int = 0, seed: int = 100):
    """(params, [c]) of the binary spinodal run (seed 100: the golden 1000-step run)."""
    return binary(n, 1e-3, 0.01, 0.005, 0.2, precision), [fields.spinodal_binary(n, seed)]


def ternary_spinodal(n: int = 512, precision: int = 0, seed: int = 101, dt: float = 5e-5):
    """(params, [c1, c2]) of the ternary spinodal run (seed 101: the golden 2000-step run)."""
    return ternary(n, dt, 0.01, 0.005, 0.2, 0.3, 0.25, precision), list(fields.spinodal_ternary(n, seed))


def binary_kolmogorov(n: int = 4096, precision: int = 1, dt: float = 2e-6, coef_mode: int = 1):
    """(params, c, omega_hat) of the forced 4096^2 drop run."""
    p = binary(n, dt, 1e-3, 1e-3, 0.1, precision, coef_mode, force_amp=1.0, force_k=4.0)
    c0 = fields.drops_binary(n, 42, ndrops=64, radius=0.3, lx=p["lx"], epsilon=p["epsilon"])
    w0 = fields.random_vorticity_hat(n, 43, kmax=8.0, rms=0.1, lx=p["lx"])
    return p, c0, w0


def binary_adjoint(n: int = 512, precision: int = 0, dt: float = 1e-4, seed: int = 2024):
    """(params, c) of the adjoint setting: spinodal noise phi = U[-0.05, 0.05] minus
    its mean, c = (1 + phi) / 2, numpy's seeded generator."""
    noise = np.random.default_rng(seed).uniform(-0.05, 0.05, (n, n))
    return binary(n, dt, 0.01, 0.005, 0.2, precision), 0.5 * (1.0 + noise - noise.mean())


ENSEMBLE_GROUPS = ((256, 32, 1e-4), (512, 24, 2.5e-5), (1024, 8, 3e-6))  # (n, members, dt)


def draw_sigmas(rng):
    """sigma_12, sigma_13, sigma_23 ~ U[0.15, 0.35], redrawn until every spreading
    coefficient gamma_i (main.c:166-170) is >= 0.1: a draw with gamma_i near or
    below 0 is an ill-posed (negative surface tension) run."""
    while True:
        s12, s13, s23 = rng.uniform(0.15, 0.35, 3)
        if min(s12 + s13 - s23, s12 + s23 - s13, s13 + s23 - s12) >= 0.1:
            return float(s12), float(s13), float(s23)


def ternary_ensemble(seed: int = 3000, precision: int = 1):
    """[(params, (c1, c2))] of the 64 ensemble members; dt per size so that the
    explicit chemical-potential term (growing as n^3 / gamma_min) stays stable."""
    rng = np.random.default_rng(seed)
    out = []
    for n, count, dt in ENSEMBLE_GROUPS:
        for _ in range(count):
            s12, s13, s23 = draw_sigmas(rng)
            p = ternary(n, dt, 0.01, 0.005, s12, s13, s23, precision)
            ph = (1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n)), 1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n)))
            out.append((p, ph))
    return out
