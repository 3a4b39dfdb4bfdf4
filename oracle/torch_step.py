"""Differentiable restatement of the reference step in torch (FP64, CPU) -- test
infrastructure only.

This module restates, with torch operations on the host, the same arithmetic as
oracle/chns_oracle.c: the ETD2RK step of the pure Navier-Stokes, binary and
ternary models (etd2rk.c:14-224 with coef_mode 1: expm1 / series coefficients), the
right-hand sides of nonlin.c:13-381, surface_tension.c:13-227 and
chem_potential.c:12-94, and the final-time loss built from free_energy.c:3-157
(pure Navier-Stokes: the kinetic energy of kinetic_energy.c and the enstrophy).  torch's reverse mode then
gives the exact gradient of the discrete map, which is the checker of the
hand-written discrete adjoint (chns_adjoint): same loss, same gradients with
respect to the stored real and imaginary parts of the initial spectral state and
to the parameters (nu), (nu, lambda, sigma) or (nu, lambda, sigma_12, sigma_13, sigma_23).

It is pinned on the CPU against the C restatement (forward, to round-off) and
against central differences of the C restatement (gradients), and it writes the
golden gradients of tests/golden/adjoint_*.npz (tests/golden/make_adjoint_golden.py).

Only tests/ may import this module.  Nothing in the product imports it.

Conventions (the reference's): spectral fields are (nx, ny/2 + 1) complex in
FFTW's r2c layout, x the slow index; dfft is the unnormalised r2c transform
(fft.c:11-14), ifft the c2r transform scaled by 1/(nx ny) (fft.c:16-31), which
ignores the imaginary parts of the ky = 0 and ky = ny/2 columns of the last
dimension as FFTW does; kx is Nyquist-positive (functions.c:11-33); the
truncation is the sharp cut k^2 > ((nx / dealias_div) (2 pi / lx))^2
(functions.c:47-84).
"""
from __future__ import annotations

import math

import torch

DT = torch.float64


class TorchStep:
    """The reference step of one configuration (dict as for oracle.Oracle)."""

    def __init__(self, p: dict):
        if p.get("coef_mode", 0) != 1:
            raise ValueError("the differentiable step restates coef_mode 1 (expm1 / series coefficients)")
        if p["model"] not in (0, 1, 2):
            raise ValueError("pure Navier-Stokes (0), binary (1) or ternary (2) model")
        self.p = dict(p)
        self.model = p["model"]
        nx, ny = p["nx"], p["ny"]
        self.nx, self.ny = nx, ny
        fx, fy = 2 * math.pi / p["lx"], 2 * math.pi / p["ly"]
        kx = torch.tensor([fx * (i if i <= nx // 2 else i - nx) for i in range(nx)], dtype=DT)
        ky = torch.tensor([fy * j for j in range(ny // 2 + 1)], dtype=DT)
        self.kx, self.ky = kx[:, None], ky[None, :]
        self.ks = self.kx * self.kx + self.ky * self.ky
        dax = (nx / p.get("dealias_div", 4.0)) * fx  # functions.c:56-59: only the x extent
        self.keep = (self.ks <= dax * dax).to(DT)
        self.dt = float(p["dt"])
        self.eps = float(p.get("epsilon", 0.0))
        self.xlambda = float(p.get("xlambda", 2.0))
        # vorticity of the Kolmogorov forcing F0 sin(kf y) x-hat, -F0 kf cos(kf y),
        # transformed like any field (the C restatement's extension)
        self.forc = None
        if p.get("force_amp", 0.0) != 0.0:
            y = torch.arange(ny, dtype=DT) * (p["ly"] / ny)
            row = -p["force_amp"] * p["force_k"] * torch.cos(p["force_k"] * y)
            self.forc = torch.fft.rfft2(row[None, :].expand(nx, ny).contiguous())

    # --- transforms and spectral helpers (fft.c, functions.c, velocity.c, curl.c)
    def dfft(self, x):
        return torch.fft.rfft2(x)

    def ifft(self, a):
        return torch.fft.irfft2(a, s=(self.nx, self.ny))

    def T(self, a):
        return a * self.keep

    def ikx(self, a):
        return 1j * self.kx * a

    def iky(self, a):
        return 1j * self.ky * a

    def velocity(self, w):
        pos = self.ks > 1e-12
        psi = torch.where(pos, w / torch.where(pos, self.ks, torch.ones_like(self.ks)), torch.zeros_like(w))
        return 1j * self.ky * psi, -1j * self.kx * psi

    def curl(self, ux, uy):
        return 1j * (self.kx * uy - self.ky * ux)

    # --- parameters
    def params(self, prm: dict) -> dict:
        """prm holds 0-d tensors: nu, lambda, sigma (binary) or nu, lambda, sigma12,
        sigma13, sigma23 (ternary); adds the derived gamma_i and Delta
        (main.c:166-170)."""
        q = dict(prm)
        if self.model == 2:
            s12, s13, s23 = q["sigma12"], q["sigma13"], q["sigma23"]
            q["g1"] = s12 - s23 + s13
            q["g2"] = s12 - s13 + s23
            q["g3"] = s23 - s12 + s13
            g1, g2, g3 = q["g1"], q["g2"], q["g3"]
            q["del"] = 6.0 * g1 * g2 * g3 / (g1 * g2 + g1 * g3 + g2 * g3)
        return q

    # --- right-hand sides
    def rhs(self, w, c1, c2, q):
        """N(omega), N(c1)[, N(c2)] (potential() + nonlin(), etd2rk.c:28,40-51)."""
        T, ifft, dfft = self.T, self.ifft, self.dfft
        eps, ks = self.eps, self.ks
        ux, uy = self.velocity(w)
        uxr, uyr = ifft(T(ux)), ifft(T(uy))
        # -(u . grad) omega  (nonlin.c:30-101)
        nw = -dfft(uxr * ifft(T(self.ikx(w))) + uyr * ifft(T(self.iky(w))))
        if self.forc is not None:
            nw = nw + self.forc
        if self.model == 0:
            return nw, None, None
        lam = q["lambda"]
        if self.model == 1:
            sg = q["sigma"]
            cr = ifft(T(c1))
            fhat = dfft(cr * (1.0 - cr) * (1.0 - 2.0 * cr))
            # mu = 1.5 sigma eps k^2 c + 24 (sigma/eps) F[f(c)]  (surface_tension.c:19-57)
            mu = (1.5 * sg * eps) * ks * c1 + (24.0 * sg / eps) * fhat
            mur = ifft(T(mu))
            nw = nw + self.curl(dfft(ifft(T(self.ikx(c1))) * mur), dfft(ifft(T(self.iky(c1))) * mur))
            # Cahn-Hilliard right-hand side (nonlin.c:174-254)
            adv = dfft(uxr * ifft(T(self.ikx(c1))) + uyr * ifft(T(self.iky(c1))))
            n1 = -adv - lam * ((24.0 * sg / eps) * ks * fhat)
            return nw, n1, None
        g1, g2, g3 = q["g1"], q["g2"], q["g3"]
        # chem_potential.c:12-94
        a, b = ifft(T(c1)), ifft(T(c2))
        d = 1.0 - a - b
        abd = a * b * d
        six = 6.0 * self.xlambda
        G1 = g1 * (a * (1.0 - a) * (1.0 - 2.0 * a)) + six * abd * b * d
        G2 = g2 * (b * (1.0 - b) * (1.0 - 2.0 * b)) + six * abd * a * d
        G3 = g3 * (d * (1.0 - d) * (1.0 - 2.0 * d)) + six * abd * a * b
        fac = 2.0 * q["del"] / eps
        muF1 = dfft(((G1 - G2) / g2 + (G1 - G3) / g3) * fac)
        muF2 = dfft(((G2 - G1) / g1 + (G2 - G3) / g3) * fac)
        # surface_tension.c:114-225
        A = muF1 + (0.75 * g1 * eps) * ks * c1
        B = muF2 + (0.75 * g2 * eps) * ks * c2
        Ar, Br = ifft(T(A)), ifft(T(B))
        m1 = (1.0 + g3 / g1) * Ar + (g3 / g2) * Br
        m2 = (g3 / g1) * Ar + (1.0 + g3 / g2) * Br
        nw = nw + self.curl(dfft(ifft(T(self.ikx(c1))) * m1), dfft(ifft(T(self.iky(c1))) * m1))
        nw = nw + self.curl(dfft(ifft(T(self.ikx(c2))) * m2), dfft(ifft(T(self.iky(c2))) * m2))
        # nonlin.c:256-377
        n1 = -dfft(ifft(T(self.ikx(c1))) * uxr + ifft(T(self.iky(c1))) * uyr) - (lam / g1) * ks * muF1
        n2 = -dfft(ifft(T(self.ikx(c2))) * uxr + ifft(T(self.iky(c2))) * uyr) - (lam / g2) * ks * muF2
        return nw, n1, n2

    # --- ETD2RK (etd2rk.c:81-212), coef_mode 1
    def _phi1(self, z):
        """dt (e^z - 1) / z, dt at z = 0."""
        zero = z == 0
        zs = torch.where(zero, torch.ones_like(z), z)
        return torch.where(zero, torch.full_like(z, self.dt), self.dt * (torch.expm1(zs) / zs))

    def _phi2(self, z):
        """dt (e^z - 1 - z) / z^2: the series sum_n z^n / (n + 2)! (20 terms) where
        |z| < 0.5, the closed form elsewhere."""
        small = z.abs() < 0.5
        zsm = torch.where(small, z, torch.zeros_like(z))
        term = torch.full_like(z, 0.5)
        acc = term
        for n in range(1, 20):
            term = term * zsm / float(n + 2)
            acc = acc + term
        zl = torch.where(small, torch.ones_like(z), z)
        closed = (torch.expm1(zl) - zl) / (zl * zl)
        return self.dt * torch.where(small, acc, closed)

    def coefs(self, q):
        dt, ks = self.dt, self.ks
        zw = (-q["nu"] * ks) * dt
        eta = torch.exp(-q["nu"] * dt * ks)
        if self.model == 0:
            return eta, self._phi1(zw), self._phi2(zw), None, None, None
        if self.model == 1:
            cc = -1.5 * q["lambda"] * q["sigma"] * self.eps * ks * ks
        else:
            cc = (-0.75 * q["lambda"] * self.eps) * (ks * ks)
        zc = dt * cc
        return eta, self._phi1(zw), self._phi2(zw), torch.exp(dt * cc), self._phi1(zc), self._phi2(zc)

    def step(self, state, q):
        eta, z1w, z2w, beta, z1c, z2c = self.coefs(q)
        if self.model == 0:
            w = state[0]
            nw0 = self.rhs(w, None, None, q)[0]
            w1 = w * eta + nw0 * z1w
            nw1 = self.rhs(w1, None, None, q)[0]
            return [w1 + (nw1 - nw0) * z2w]
        w, c1 = state[0], state[1]
        c2 = state[2] if self.model == 2 else None
        nw0, n10, n20 = self.rhs(w, c1, c2, q)
        w1 = w * eta + nw0 * z1w
        c11 = c1 * beta + n10 * z1c
        c21 = c2 * beta + n20 * z1c if c2 is not None else None
        nw1, n11, n21 = self.rhs(w1, c11, c21, q)
        out = [w1 + (nw1 - nw0) * z2w, c11 + (n11 - n10) * z2c]
        if c2 is not None:
            out.append(c21 + (n21 - n20) * z2c)
        return out

    def run(self, state, q, nsteps: int):
        for _ in range(nsteps):
            state = self.step(state, q)
        return state

    # --- the loss at the final state (free_energy.c:3-157; c, grad c untruncated)
    def loss(self, state, prm: dict, weights=(1.0, 1.0, 1.0)):
        q = self.params(prm)
        eps = self.eps
        ifft = self.ifft
        if self.model == 0:
            # kinetic energy of the truncated velocity (kinetic_energy.c:17-21,43-49,89)
            # and the enstrophy of the truncated vorticity
            ux, uy = self.velocity(state[0])
            u, v = ifft(self.T(ux)), ifft(self.T(uy))
            wt = ifft(self.T(state[0]))
            return weights[0] * torch.mean(0.5 * (u * u + v * v)) + weights[1] * torch.mean(0.5 * wt * wt)
        if self.model == 1:
            ch = state[1]
            c = ifft(ch)
            cx, cy = ifft(self.ikx(ch)), ifft(self.iky(ch))
            sg = q["sigma"]
            eb = torch.mean(12.0 * (sg / eps) * c * c * (1.0 - c) * (1.0 - c))
            g2 = torch.mean(cx * cx + cy * cy)
            return weights[0] * eb + weights[1] * (0.75 * sg * eps) * g2 + weights[2] * 4.0 * g2
        g1, g2, g3 = q["g1"], q["g2"], q["g3"]
        c1h, c2h = state[1], state[2]
        c1, c2 = ifft(c1h), ifft(c2h)
        c1x, c1y = ifft(self.ikx(c1h)), ifft(self.iky(c1h))
        c2x, c2y = ifft(self.ikx(c2h)), ifft(self.iky(c2h))
        c3 = 1.0 - c1 - c2
        eb = (6.0 / eps) * torch.mean(g1 * c1 ** 2 * (1 - c1) ** 2 + g2 * c2 ** 2 * (1 - c2) ** 2
                                      + g3 * c3 ** 2 * (c1 + c2) ** 2)
        eg = 0.375 * eps * torch.mean(g1 * (c1x ** 2 + c1y ** 2) + g2 * (c2x ** 2 + c2y ** 2)
                                      + g3 * ((c1x + c2x) ** 2 + (c1y + c2y) ** 2))
        gp = torch.mean(c1x ** 2 + c1y ** 2 + c2x ** 2 + c2y ** 2)
        return weights[0] * eb + weights[1] * eg + weights[2] * gp


PARAM_NAMES = {0: ("nu",), 1: ("nu", "lambda", "sigma"), 2: ("nu", "lambda", "sigma12", "sigma13", "sigma23")}


def forward(p: dict, state, nsteps: int):
    """Final state (numpy complex arrays) after nsteps steps from `state`."""
    import numpy as np

    ts = TorchStep(p)
    prm = {k: torch.tensor(float(p[k]), dtype=DT) for k in PARAM_NAMES[p["model"]]}
    with torch.no_grad():
        out = ts.run([torch.from_numpy(np.ascontiguousarray(s, np.complex128)) for s in state],
                     ts.params(prm), nsteps)
    return [o.numpy() for o in out]


def gradient(p: dict, state, nsteps: int, weights=(1.0, 1.0, 1.0)):
    """J and its gradients after nsteps steps from `state`: (J, g_w, [g_c1, g_c2], g_params),
    the state gradients with respect to the stored real and imaginary parts
    (g = dJ/dRe + i dJ/dIm), g_params in PARAM_NAMES order."""
    import numpy as np

    ts = TorchStep(p)
    names = PARAM_NAMES[p["model"]]
    prm = {k: torch.tensor(float(p[k]), dtype=DT, requires_grad=True) for k in names}
    st0 = [torch.from_numpy(np.ascontiguousarray(s, np.complex128).copy()).requires_grad_(True) for s in state]
    fin = ts.run(list(st0), ts.params(prm), nsteps)
    J = ts.loss(fin, prm, weights)
    grads = torch.autograd.grad(J, st0 + [prm[k] for k in names])
    ns = len(st0)
    return (float(J.detach()), grads[0].numpy(), [g.numpy() for g in grads[1:ns]],
            np.array([float(g) for g in grads[ns:]]))
