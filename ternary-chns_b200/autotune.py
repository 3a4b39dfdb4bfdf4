#!/usr/bin/env python3
"""Autotuner of the launch shapes of the step and transform kernels (csrc/chns_tuned.h).

Three choices per grid size and precision, each timed on forward binary and
ternary steps (the candidate with the highest summed steps/s wins):

* threads per CTA (``threads`` pass).  Every row and column kernel runs n/16
  threads per transform of n points and packs several transforms into one CTA.
  Few threads per CTA spread the rows of a small grid over all SMs; more threads
  share twiddles and give wider tile loads on large grids.  The CTA shape is a
  template argument, so this pass builds one library variant per candidate
  (-DCHNS_CTA_THREADS=T) and times it in a fresh process.
* rows per TMA box of the row kernels' tiles (``box`` pass, 64 / 128 / 256): a
  tile is whole boxes, so smaller boxes fetch fewer zero rows beyond the cut and
  take less shared memory, for more copies per tile.
* the P1 split (``split`` pass): the spectral inverse pass with two CTAs per row
  (half the outputs each) or one.
* P4's grad c (``grad`` pass): kept in real space by P2 (one more field written
  and read per phase field) or transformed again by P4 (two more transforms per
  x-row pair and phase field).
* programmatic dependent launches of the stage kernels (``pdl`` pass): each kernel
  scheduled while the one before drains, waiting on the device for it.

The box, split, grad and pdl choices are run-time (chns_tune_override, for contexts
created afterwards), so those passes time one library.  Such a candidate replaces
the current table entry only when it is more than ``--margin`` (1%) faster, so
that run-to-run noise does not flip choices.  Results are bitwise the same under
every choice (tests/test_gpu_tuning.py).

The transforms' radix order is not a knob: a thread holds 16 elements, so every
stage but one is radix 16, the remaining radix-2/4/8 stage must come first (the
last stage leaves the result in registers in natural order), and moving it
changes the twiddle multiplies by at most one per thread and stage.

Passes not run keep the values of the current header.  It needs a GPU:

    python ternary-chns_b200/autotune.py --passes threads,box,split,grad,pdl \\
        --out ternary-chns_b200/csrc/chns_tuned.h --report autotune.json
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
TUNED = os.path.join(HERE, "csrc", "chns_tuned.h")
THREADS = [32, 64, 128, 256]
BOX_ROWS = [64, 128, 256]
SPLIT = [0, 1]
GRAD = [0, 1]
PDL = [0, 1]
TIMED_SIZES = [256, 512, 1024, 2048, 4096]
ALL_SIZES = [32, 64, 128, 256, 512, 1024, 2048, 4096]
TABLES = ["kCtaThreads", "kTmaBoxRows", "kSpecInvSplit", "kP4Grad", "kPdl"]


def time_variant(lib: str, box: int = -1, split: int = -1, grad: int = -1, pdl: int = -1, steps_small: int = 200,
                 steps_large: int = 40) -> dict:
    """Steps/s of each (model, n, precision) with the library at `lib` and the
    given run-time overrides (-1: the tuned table)."""
    import numpy as np

    sys.path.insert(0, HERE)
    import chns_b200 as C

    C.load_library(lib)
    C.tune_override(C.TUNE_TMA_BOX_ROWS, box)
    C.tune_override(C.TUNE_P1_SPLIT, split)
    C.tune_override(C.TUNE_P4_GRAD, grad)
    C.tune_override(C.TUNE_PDL, pdl)
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
    C.tune_override(C.TUNE_TMA_BOX_ROWS, -1)
    C.tune_override(C.TUNE_P1_SPLIT, -1)
    C.tune_override(C.TUNE_P4_GRAD, -1)
    C.tune_override(C.TUNE_PDL, -1)
    return out


def read_tables(path: str = TUNED) -> dict:
    """{(table, prec): [8 values]} of a tuned header (prec 0 = F64, 1 = F32)."""
    text = open(path).read()
    out = {}
    for name in TABLES:
        for prec, suf in ((0, "F64"), (1, "F32")):
            m = re.search(rf"{name}{suf}\[8\]\s*=\s*\{{([^}}]*)\}}", text)
            out[(name, prec)] = [int(v) for v in m.group(1).split(",")]
    return out


def header(t: dict) -> str:
    def row(name, prec):
        return ", ".join(str(v) for v in t[(name, prec)])

    return f"""// chns_tuned.h -- launch shapes of the step and transform kernels for each grid
// size and precision (index log2(n) - 5, n = 32 .. 4096): threads per CTA, TMA box
// rows, the P1 split, the source of P4's grad c and programmatic dependent
// launches of the stage kernels.  Chosen by ternary-chns_b200/autotune.py from
// forward-step timings of the binary and ternary models on a B200: the candidate
// with the highest summed steps/s.  Each CTA runs threads / (n/16) transforms of
// n points side by side; small grids want few threads per CTA so that the rows
// spread over all 148 SMs.
#pragma once

namespace chns {{

constexpr int kCtaThreadsF64[8] = {{{row("kCtaThreads", 0)}}};
constexpr int kCtaThreadsF32[8] = {{{row("kCtaThreads", 1)}}};

// Rows per TMA box of the row kernels' tiles (a tile is whole boxes, so smaller
// boxes over-fetch fewer zero rows beyond the cut at the price of more copies).
constexpr int kTmaBoxRowsF64[8] = {{{row("kTmaBoxRows", 0)}}};
constexpr int kTmaBoxRowsF32[8] = {{{row("kTmaBoxRows", 1)}}};

// P1 with two CTAs per row (each half of the outputs): 1 = on.
constexpr int kSpecInvSplitF64[8] = {{{row("kSpecInvSplit", 0)}}};
constexpr int kSpecInvSplitF32[8] = {{{row("kSpecInvSplit", 1)}}};

// grad c_i kept in real space from P2 for P4 (1), or transformed again by P4 (0).
constexpr int kP4GradF64[8] = {{{row("kP4Grad", 0)}}};
constexpr int kP4GradF32[8] = {{{row("kP4Grad", 1)}}};

// stage kernels launched as programmatic dependent launches (1), or plainly (0).
constexpr int kPdlF64[8] = {{{row("kPdl", 0)}}};
constexpr int kPdlF32[8] = {{{row("kPdl", 1)}}};

}}  // namespace chns
"""


def _time_in_process(lib: str, box: int = -1, split: int = -1, grad: int = -1, pdl: int = -1) -> dict:
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--time", lib, "--box", str(box),
                        "--split", str(split), "--grad", str(grad), "--pdl", str(pdl)], capture_output=True,
                       text=True, check=True)
    return json.loads(r.stdout.strip().splitlines()[-1])


def _score(res: dict, n: int, prec: int) -> float:
    return sum(res[f"{m}/{n}/{prec}"] for m in (1, 2))


def _pick(results: dict, table: list, prec: int, margin: float, allowed=lambda cand, n: True) -> list:
    """New table: per timed size the best candidate, kept at the current value
    unless the best beats it by more than `margin` (when the current value was timed)."""
    out = list(table)
    for n in TIMED_SIZES:
        li = ALL_SIZES.index(n)
        score = {cand: _score(res, n, prec) for cand, res in results.items() if allowed(cand, n)}
        best = max(score, key=score.get)
        cur = table[li]
        if cur in score and score[best] <= score[cur] * (1 + margin):
            best = cur
        out[li] = best
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--passes", default="threads,box,split,grad,pdl",
                    help="comma list of threads, box, split, grad, pdl")
    ap.add_argument("--out", required=False, help="header to write")
    ap.add_argument("--report", help="also write the measured tables (JSON) here")
    ap.add_argument("--margin", type=float, default=0.01, help="gain a run-time choice's change needs")
    ap.add_argument("--lib", help="library the box and split passes time (default: the in-tree build)")
    ap.add_argument("--time", help="(internal) time one library variant and print JSON")
    ap.add_argument("--box", type=int, default=-1, help="(internal) box-rows override of --time")
    ap.add_argument("--split", type=int, default=-1, help="(internal) P1-split override of --time")
    ap.add_argument("--grad", type=int, default=-1, help="(internal) P4-grad override of --time")
    ap.add_argument("--pdl", type=int, default=-1, help="(internal) PDL override of --time")
    a = ap.parse_args()
    if a.time:
        print(json.dumps(time_variant(a.time, a.box, a.split, a.grad, a.pdl)))
        return
    sys.path.insert(0, HERE)
    import build as B

    passes = [p for p in a.passes.split(",") if p]
    tables = read_tables()
    report = {}
    if "threads" in passes:
        results = {}
        with tempfile.TemporaryDirectory() as tmp:
            for t in THREADS:
                lib = os.path.join(tmp, f"t{t}", "libchns_b200.so")
                B.build(defines=(f"CHNS_CTA_THREADS={t}",), build_dir=os.path.join(tmp, f"b{t}"), lib=lib)
                results[t] = _time_in_process(lib)
                print(f"threads {t}:", json.dumps(results[t]), flush=True)
        for prec in (0, 1):
            # a transform needs n/16 threads: a smaller candidate runs as one transform per CTA
            tables[("kCtaThreads", prec)] = _pick(results, tables[("kCtaThreads", prec)], prec, 0.0,
                                                  lambda t, n: t >= n // 16 or t == THREADS[-1])
        report["threads"] = {str(k): v for k, v in results.items()}
    lib = a.lib or B.LIB
    if not os.path.isfile(lib):
        raise SystemExit(f"{lib} is missing: build the library first (build.py)")
    if "box" in passes:
        results = {b: _time_in_process(lib, box=b) for b in BOX_ROWS}
        for prec in (0, 1):
            tables[("kTmaBoxRows", prec)] = _pick(results, tables[("kTmaBoxRows", prec)], prec, a.margin)
        report["box"] = {str(k): v for k, v in results.items()}
        print("box:", json.dumps(report["box"]), flush=True)
    if "split" in passes:
        results = {s: _time_in_process(lib, split=s) for s in SPLIT}
        for prec in (0, 1):
            tables[("kSpecInvSplit", prec)] = _pick(results, tables[("kSpecInvSplit", prec)], prec, a.margin)
        report["split"] = {str(k): v for k, v in results.items()}
        print("split:", json.dumps(report["split"]), flush=True)
    if "grad" in passes:
        results = {g: _time_in_process(lib, grad=g) for g in GRAD}
        for prec in (0, 1):
            tables[("kP4Grad", prec)] = _pick(results, tables[("kP4Grad", prec)], prec, a.margin)
        report["grad"] = {str(k): v for k, v in results.items()}
        print("grad:", json.dumps(report["grad"]), flush=True)
    if "pdl" in passes:
        results = {q: _time_in_process(lib, pdl=q) for q in PDL}
        for prec in (0, 1):
            tables[("kPdl", prec)] = _pick(results, tables[("kPdl", prec)], prec, a.margin)
        report["pdl"] = {str(k): v for k, v in results.items()}
        print("pdl:", json.dumps(report["pdl"]), flush=True)
    text = header(tables)
    if a.out:
        with open(a.out, "w") as f:
            f.write(text)
    if a.report:
        report["chosen"] = {f"{k[0]}/{k[1]}": v for k, v in tables.items()}
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)
    print(text)


if __name__ == "__main__":
    main()
