"""Seeded synthetic initial fields (no dataset is involved anywhere on this path).

All generators are deterministic functions of an integer seed: splitmix64 ->
uniform doubles in [0, 1), so the oracle and the GPU see the same bits.
Real fields are (nx, ny) float64 arrays, row i = x index, as read by the
reference's read_array_real (read_array.c:20-29).
"""
from __future__ import annotations

import math

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def uniform(seed: int, n: int) -> np.ndarray:
    """n uniform doubles in [0, 1) from splitmix64 seeded with `seed`."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + (np.arange(1, n + 1, dtype=np.uint64) * _GOLDEN)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def spinodal_binary(n: int, seed: int, amp: float = 0.05) -> np.ndarray:
    """Binary spinodal start: phi = U[-amp, amp] minus its mean, c = (1 + phi) / 2."""
    phi = (2.0 * uniform(seed, n * n) - 1.0) * amp
    phi -= phi.mean()
    return (0.5 * (1.0 + phi)).reshape(n, n)


def spinodal_ternary(n: int, seed: int, amp: float = 0.02):
    """Ternary start: c_i = 1/3 + U[-amp, amp] for i = 1, 2 (c3 = 1 - c1 - c2)."""
    u = uniform(seed, 2 * n * n)
    c1 = 1.0 / 3.0 + (2.0 * u[: n * n] - 1.0) * amp
    c2 = 1.0 / 3.0 + (2.0 * u[n * n:] - 1.0) * amp
    return c1.reshape(n, n), c2.reshape(n, n)


def drops_binary(n: int, seed: int, ndrops: int = 64, radius: float = 0.3, lx: float = 2 * math.pi,
                 epsilon: float | None = None) -> np.ndarray:
    """Drops of c = 1 on c = 0 with the reference's tanh profile
    c = (1 - tanh((r - R) / (0.5 eps))) / 2 (init.c:236-242), at seeded uniform
    centres, periodic distance; overlapping drops take the maximum."""
    if epsilon is None:
        epsilon = 2.0 * (lx / n)
    u = uniform(seed, 2 * ndrops)
    cx, cy = u[:ndrops] * lx, u[ndrops:] * lx
    x = np.arange(n) * (lx / n)
    c = np.zeros((n, n))
    for k in range(ndrops):
        dxv = np.abs(x - cx[k]); dxv = np.minimum(dxv, lx - dxv)
        dyv = np.abs(x - cy[k]); dyv = np.minimum(dyv, lx - dyv)
        r = np.sqrt(dxv[:, None] ** 2 + dyv[None, :] ** 2)
        c = np.maximum(c, 0.5 * (1.0 - np.tanh((r - radius) / (0.5 * epsilon))))
    return c


def random_vorticity_hat(n: int, seed: int, kmax: float = 8.0, rms: float = 0.1, lx: float = 2 * math.pi):
    """Spectral vorticity (FFTW layout n x (n/2+1), unnormalised) with random
    phases and unit amplitudes on modes 0 < |k| <= kmax, scaled to real-space rms."""
    f = 2 * math.pi / lx
    kx = np.where(np.arange(n) <= n // 2, np.arange(n), np.arange(n) - n) * f
    ky = np.arange(n // 2 + 1) * f
    k = np.sqrt(kx[:, None] ** 2 + ky[None, :] ** 2)
    mask = (k > 0) & (k <= kmax)
    ph = uniform(seed, mask.size).reshape(mask.shape)
    w = np.where(mask, np.exp(2j * math.pi * ph), 0.0)
    # make the ky = 0 column Hermitian so the field is real
    for i in range(1, n // 2):
        w[n - i, 0] = np.conj(w[i, 0])
    w[0, 0] = 0.0
    real = np.fft.irfft2(w, s=(n, n))
    s = rms / max(np.sqrt(np.mean(real ** 2)), 1e-300)
    return (w * s).astype(np.complex128)
