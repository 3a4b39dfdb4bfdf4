#!/usr/bin/env python3
"""Generates tests/golden/adjoint_bin64.npz, adjoint_ter64.npz and adjoint_ns32.npz:
the loss and its exact gradients after 12 ETD2RK steps from the bin64 / ter64 / ns32
initial states
(coef_mode 1), computed by reverse mode through oracle/torch_step.py (a torch
restatement of the reference step, pinned on the CPU against the C restatement
and against its central differences by tests/test_oracle_adjoint.py).

These are the golden gradients for the discrete adjoint chns_adjoint (all loss
weights 1): g_w = dJ/d(omega_hat_0), g_c = dJ/d(c_hat_0) (binary), dJ/d(c1_hat_0),
dJ/d(c2_hat_0) (ternary) or none (pure Navier-Stokes), each with respect to the
stored real and imaginary parts (g = dJ/dRe + i dJ/dIm), and g_params = dJ/d(nu,
lambda, sigma), dJ/d(nu, lambda, sigma_12, sigma_13, sigma_23) or dJ/d(nu).

Usage:  python tests/golden/make_adjoint_golden.py [case ...]   (default: every case)
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

STEPS = 12
CASES = ("bin64", "ter64", "ns32")


def case(name: str):
    """(params, initial state) of an adjoint golden case."""
    from _golden import load_small

    g = load_small(name)
    return dict(g["params"], coef_mode=1), [np.asarray(s) for s in g["init"]]


def compute(name: str) -> dict:
    import torch_step as TS

    p, init = case(name)
    J, gw, gcs, gp = TS.gradient(p, init, STEPS)
    g_c = np.stack(gcs) if gcs else np.zeros((0,) + gw.shape, gw.dtype)
    return {"params": json.dumps(p), "steps": STEPS, "J": J, "g_w": gw, "g_c": g_c,
            "g_params": gp, "param_names": json.dumps(list(TS.PARAM_NAMES[p["model"]]))}


def main(names=None):
    for name in names or CASES:
        out = os.path.join(HERE, f"adjoint_{name}.npz")
        np.savez_compressed(out, **compute(name))
        print("wrote", out)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
