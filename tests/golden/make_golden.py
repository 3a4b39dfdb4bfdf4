#!/usr/bin/env python3
"""Generates the golden fixtures in tests/golden/ by running the REFERENCE's own
compiled sources (oracle/_ref/<config>/libref.so, built by oracle/build_ref.py).

The reference ships no tests, fixtures or golden vectors of its own, so these
vectors are the reference run here: its etd2rk.c / nonlin.c / ... code, with the
oracle's FP64 FFT behind its FFTW calls.  They pin both the C restatement
(oracle/chns_oracle.c) and, through it, the GPU path.

Small grids store full spectral states; the two full-size configurations
(binary 256^2 x 1000 steps, ternary 512^2 x 2000 steps) store the full final
spectral state (1 MB and 6.3 MB) beside a fingerprint of it (see fingerprint());
the big grids (4096^2, 1024^2) store only the fingerprint.

The reference's source folder is taken from CHNS_REFERENCE_DIR (oracle/build_ref.py).

Usage:  python tests/golden/make_golden.py [--full] [--big] [--init] [--only] [--names a,b]
  (--init: only init_ref.npz; --only: skip the small fixtures and init_ref.npz;
  --names: only the named small fixtures)
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "ternary-chns_b200"))

from chns_b200 import fields  # noqa: E402

# scenario: (config, steps, phase seed, vorticity seed or None, vorticity kmax, rms)
SMALL = [
    ("ns32", 20, None, 3, 6.0, 1.0),
    ("bin32", 20, 1, 5, 6.0, 0.5),
    ("bin64", 20, 1, 5, 6.0, 0.5),
    ("ter32", 20, 2, 5, 6.0, 0.5),
    ("ter64", 20, 2, 5, 6.0, 0.5),
    ("bindef64", 20, 4, 6, 3.0, 0.5),
    ("terdef64", 20, 4, 6, 3.0, 0.5),
    # SMOOTH_FILTER builds of the reference
    ("nssf32", 20, None, 3, 6.0, 1.0),
    ("binsf64", 20, 1, 5, 6.0, 0.5),
    ("tersf64", 20, 2, 5, 6.0, 0.5),
    ("binsfdef64", 20, 4, 6, 3.0, 0.5),
]
FULL = [
    # binary spinodal run: 256^2, omega = 0, c = (1 + U(+-0.05) - mean)/2, 1000 steps
    ("bin256", 1000, 100, None, 0.0, 0.0),
    # ternary spinodal run: 512^2, omega = 0, c_i = 1/3 + U(+-0.02), 2000 steps at dt = 5e-5
    ("ter512", 2000, 101, None, 0.0, 0.0),
]

# large grids, a few steps from spinodal noise plus random low-k vorticity: parity of
# the 1024^2 / 4096^2 kernels (the same fingerprint as FULL)
BIG = [
    ("bin4096", 2, 102, 103, 8.0, 0.1),
    ("ter1024", 3, 104, 105, 8.0, 0.1),
]

NPROJ = 8
KLOW = 16


def initial_state(model: int, n: int, lx: float, phase_seed, w_seed, kmax, rms):
    """Returns (real phase fields, omega_hat) of a scenario."""
    p1 = p2 = None
    if model == 1:
        p1 = fields.spinodal_binary(n, phase_seed)
    elif model == 2:
        p1, p2 = fields.spinodal_ternary(n, phase_seed)
    w = None
    if w_seed is not None:
        w = fields.random_vorticity_hat(n, w_seed, kmax=kmax, rms=rms, lx=lx)
    return p1, p2, w


def apply_initial(sim, model, p1, p2, w):
    """init.c INIT_READ_DATA order: phase fields via dfft + truncation, omega_hat set after."""
    if model >= 1:
        sim.set_phase_real(p1, p2)
    if w is not None:
        st = sim.get_state()
        st[0] = w
        sim.set_state(*st)


def fingerprint(spec: np.ndarray, seed: int = 1000) -> dict:
    """Size-independent summary of a spectral field (n x (n/2+1) complex):
    the block |m| <= KLOW, j <= KLOW; NPROJ random projections over all modes;
    the L2 norm; the k = 0 mode."""
    n = spec.shape[0]
    rows = list(range(0, KLOW + 1)) + list(range(n - KLOW, n))
    low = spec[rows, : KLOW + 1]
    flat = spec.reshape(-1)
    proj = []
    for r in range(NPROJ):
        u = fields.uniform(seed + r, 2 * flat.size)
        wgt = (2 * u[: flat.size] - 1) + 1j * (2 * u[flat.size:] - 1)
        proj.append(np.sum(wgt * flat))
    return dict(low=low, proj=np.array(proj), norm=float(np.sqrt(np.sum(np.abs(flat) ** 2))),
                k0=complex(spec[0, 0]))


def fingerprint_rel_err(fp_ref: dict, fp: dict) -> float:
    """max over the parts of ||part - ref|| / ||field||-scaled reference."""
    e_low = np.linalg.norm(fp["low"] - fp_ref["low"]) / max(np.linalg.norm(fp_ref["low"]), 1e-300)
    e_proj = np.linalg.norm(fp["proj"] - fp_ref["proj"]) / max(np.linalg.norm(fp_ref["proj"]), 1e-300)
    e_norm = abs(fp["norm"] - fp_ref["norm"]) / max(fp_ref["norm"], 1e-300)
    return float(max(e_low, e_proj, e_norm))


def make_small(O, names=None):
    for name, steps, ps, ws, kmax, rms in SMALL:
        if names and name not in names:
            continue
        p = O.ref_config_params(name)
        R = O.RefLib(name)
        n = p["nx"]
        p1, p2, w = initial_state(p["model"], n, p["lx"], ps, ws, kmax, rms)
        apply_initial(R, p["model"], p1, p2, w)
        s0 = R.get_state()
        r0 = R.rhs()
        R.set_state(*s0)
        fe0 = R.free_energy() if p["model"] >= 1 else (0.0, 0.0)
        ke0 = R.kinetic_energy()
        R.step(steps)
        s1 = R.get_state()
        out = dict(params=json.dumps(p), steps=steps)
        for k, a in enumerate(s0):
            out[f"init{k}"] = a
        for k, a in enumerate(r0):
            out[f"rhs{k}"] = a
        for k, a in enumerate(s1):
            out[f"final{k}"] = a
        out["fe0"] = np.array(fe0)
        out["ke0"] = np.array(ke0)
        # FFT pair of the reference's fft.c on a seeded field
        x = fields.uniform(77, n * n).reshape(n, n) - 0.5
        out["fft_in"] = x
        out["fft_dfft"] = R.dfft(x)
        out["fft_ifft"] = R.ifft(out["fft_dfft"])
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print("wrote", name)


def make_full(O, cases=None):
    for name, steps, ps, ws, kmax, rms in cases or FULL:
        p = O.ref_config_params(name)
        R = O.RefLib(name, nthreads=min(8, os.cpu_count() or 1))
        n = p["nx"]
        p1, p2, w = initial_state(p["model"], n, p["lx"], ps, ws, kmax, rms)
        apply_initial(R, p["model"], p1, p2, w)
        s0 = R.get_state()
        R.step(steps)
        s1 = R.get_state()
        out = dict(params=json.dumps(p), steps=steps)
        for k, a in enumerate(s1):
            if n <= 512:
                out[f"final{k}"] = a
            fp = fingerprint(a)
            for key, v in fp.items():
                out[f"final{k}_{key}"] = np.asarray(v)
            out[f"init{k}_k0"] = np.asarray(complex(s0[k][0, 0]))
        np.savez_compressed(os.path.join(HERE, f"{name}_fp.npz"), **out)
        print("wrote", name)


# the reference's own init() (init.c) on configurations whose macros select each branch:
# ZERO_INIT vorticity with the binary drop / ternary srand(10) noise, TG_INIT, and the
# k-space shell vorticity (neither macro)
INIT_CONFIGS = ["bin32", "ter32", "bindef64", "terdef64", "nstg32", "bintg64", "nssh32", "binsh64"]


def make_init(O):
    out = {}
    for name in INIT_CONFIGS:
        p = O.ref_config_params(name)
        R = O.RefLib(name)  # ref_setup ends with the reference's init()
        out[f"{name}_params"] = json.dumps(p)
        for k, a in enumerate(R.get_state()):
            out[f"{name}_state{k}"] = a
    np.savez_compressed(os.path.join(HERE, "init_ref.npz"), **out)
    print("wrote init_ref")


if __name__ == "__main__":
    import oracle as O
    O.build_ref.build_all()
    if "--names" in sys.argv:
        make_small(O, sys.argv[sys.argv.index("--names") + 1].split(","))
    elif "--init" in sys.argv:
        make_init(O)
    elif "--only" not in sys.argv:
        make_small(O)
        make_init(O)
    if "--full" in sys.argv:
        make_full(O)
    if "--big" in sys.argv:
        make_full(O, BIG)
