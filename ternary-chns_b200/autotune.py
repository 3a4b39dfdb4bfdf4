#!/usr/bin/env python3
"""Autotuner of the CTA shape of the step and transform kernels (csrc/chns_tuned.h).

Every row and column kernel runs n/16 threads per transform of n points and
packs several transforms into one CTA.  Few threads per CTA spread the rows of a
small grid over all SMs; more threads share twiddles and give wider tile loads
on large grids.  This script builds one library variant per candidate
(-DCHNS_CTA_THREADS=T), times the forward binary and ternary steps of every grid
size in both precisions with each variant (a fresh process per variant), and
writes the header with the fastest candidate per size and precision (highest
summed steps/s of the two models).  It needs a GPU:

    python ternary-chns_b200/autotune.py --out ternary-chns_b200/csrc/chns_tuned.h
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
CANDIDATES = [32, 64, 128, 256]
TIMED_SIZES = [256, 512, 1024, 2048, 4096]
ALL_SIZES = [32, 64, 128, 256, 512, 1024, 2048, 4096]


def time_variant(lib: str, steps_small: int = 200, steps_large: int = 40) -> dict:
    """Steps/s of each (model, n, precision) with the library at `lib`."""
    import numpy as np

    sys.path.insert(0, HERE)
    import chns_b200 as C

    C.load_library(lib)
    out = {}
    rng = np.random.default_rng(0)
    for model in (C.MODEL_BINARY, C.MODEL_TERNARY):
        for n in TIMED_SIZES:
            for prec in (C.FP64, C.FP32):
                p = C.default_params(model, n)
                p.update(precision=prec, dt=1e-6)
                steps = steps_small if n <= 1024 else steps_large
                with C.Context(p) as c:
                    if model == C.MODEL_TERNARY:
                        c.set_phase_real(1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n)),
                                         1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n)))
                    else:
                        c.set_phase_real(0.5 + 0.05 * rng.uniform(-1, 1, (n, n)))
                    c.step(10)
                    c.synchronize()
                    best = 0.0
                    for _ in range(3):
                        t0 = time.perf_counter()
                        c.step(steps)
                        c.synchronize()
                        best = max(best, steps / (time.perf_counter() - t0))
                out[f"{model}/{n}/{prec}"] = best
    return out


def header(choice: dict) -> str:
    f64 = ", ".join(str(choice[(n, 0)]) for n in ALL_SIZES)
    f32 = ", ".join(str(choice[(n, 1)]) for n in ALL_SIZES)
    return f"""// chns_tuned.h -- threads per CTA of the step and transform kernels for each
// grid size and precision (index log2(n) - 5, n = 32 .. 4096).  Chosen by
// ternary-chns_b200/autotune.py from forward-step timings of the binary and
// ternary models on a B200: the candidate with the highest summed steps/s.
// Each CTA runs threads / (n/16) transforms of n points side by side; small
// grids want few threads per CTA so that the rows spread over all 148 SMs.
#pragma once

namespace chns {{

constexpr int kCtaThreadsF64[8] = {{{f64}}};
constexpr int kCtaThreadsF32[8] = {{{f32}}};

}}  // namespace chns
"""


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=False, help="header to write")
    ap.add_argument("--time", help="(internal) time one library variant and print JSON")
    ap.add_argument("--report", help="also write the measured table (JSON) here")
    a = ap.parse_args()
    if a.time:
        print(json.dumps(time_variant(a.time)))
        return
    sys.path.insert(0, HERE)
    import build as B

    results = {}
    with tempfile.TemporaryDirectory() as tmp:
        for t in CANDIDATES:
            lib = os.path.join(tmp, f"t{t}", "libchns_b200.so")
            B.build(defines=(f"CHNS_CTA_THREADS={t}",), build_dir=os.path.join(tmp, f"b{t}"), lib=lib)
            r = subprocess.run([sys.executable, os.path.abspath(__file__), "--time", lib], capture_output=True,
                               text=True, check=True)
            results[t] = json.loads(r.stdout.strip().splitlines()[-1])
            print(f"threads {t}:", json.dumps(results[t]), flush=True)
    choice = {}
    for n in ALL_SIZES:
        for prec in (0, 1):
            if n not in TIMED_SIZES:
                choice[(n, prec)] = 32
                continue
            score = {t: sum(results[t][f"{m}/{n}/{prec}"] for m in (1, 2)) for t in CANDIDATES
                     if t >= n // 16 or t == CANDIDATES[-1]}
            choice[(n, prec)] = max(score, key=score.get)
    text = header(choice)
    if a.out:
        with open(a.out, "w") as f:
            f.write(text)
    if a.report:
        with open(a.report, "w") as f:
            json.dump({str(t): v for t, v in results.items()}, f, indent=1)
    print(text)


if __name__ == "__main__":
    main()
