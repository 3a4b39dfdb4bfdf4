"""Helpers shared by the tests: golden fixtures and scenario set-up."""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

SMALL_CONFIGS = ["ns32", "bin32", "bin64", "ter32", "ter64", "bindef64", "terdef64",
                 "nssf32", "binsf64", "tersf64", "binsfdef64"]


def load_small(name: str) -> dict:
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    out = {k: z[k] for k in z.files}
    out["params"] = json.loads(str(out["params"]))
    out["steps"] = int(out["steps"])
    model = out["params"]["model"]
    out["init"] = [out[f"init{k}"] for k in range(model + 1)]
    out["rhs"] = [out[f"rhs{k}"] for k in range(model + 1)]
    out["final"] = [out[f"final{k}"] for k in range(model + 1)]
    return out


def load_full(name: str) -> dict:
    z = np.load(os.path.join(GOLDEN, f"{name}_fp.npz"))
    out = {k: z[k] for k in z.files}
    out["params"] = json.loads(str(out["params"]))
    out["steps"] = int(out["steps"])
    return out


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
