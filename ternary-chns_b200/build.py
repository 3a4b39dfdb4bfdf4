#!/usr/bin/env python3
"""Builds libchns_b200.so (the C ABI of include/chns.h) for sm_100a with nvcc.

One translation unit per grid size is compiled in parallel, then linked with
the static CUDA runtime.  Output: ternary-chns_b200/lib/libchns_b200.so (in-tree).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUTDIR = os.path.join(HERE, "lib")
LIB = os.path.join(OUTDIR, "libchns_b200.so")
BUILD = os.path.join(HERE, "_build")
SIZES = [32, 64, 128, 256, 512, 1024, 2048, 4096]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]


def _sources():
    srcs = [os.path.join(CSRC, "chns_api.cu"), os.path.join(CSRC, "chns_noalloc.cu"),
            os.path.join(CSRC, "chns_adjoint.cu"), os.path.join(CSRC, "chns_ensemble.cu"),
            os.path.join(CSRC, "chns_init.cu"), os.path.join(CSRC, "chns_io.cu"),
            os.path.join(CSRC, "chns_diag_extra.cu"), os.path.join(CSRC, "chns_slab.cu"),
            os.path.join(CSRC, "chns_persist.cu")]
    srcs += [os.path.join(CSRC, f"chns_inst_{n}.cu") for n in SIZES]
    return srcs


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + \
        [os.path.join(ROOT, "include", "chns.h")]


def _compile(src: str, verbose: bool, build_dir: str = BUILD, defines: tuple = ()) -> str:
    obj = os.path.join(build_dir, os.path.basename(src).replace(".cu", ".o"))
    deps = [src] + _headers()
    if os.path.isfile(obj) and all(os.path.getmtime(d) <= os.path.getmtime(obj) for d in deps):
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, *[f"-D{d}" for d in defines], "-c", src, "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        with open(obj + ".ptxas.txt", "w") as f:
            f.write(r.stderr)
    return obj


def build(verbose: bool = False, jobs: int | None = None, defines: tuple = (), build_dir: str = BUILD,
          lib: str = LIB) -> str:
    """Compiles and links the library; `defines` (NAME=VALUE) and the build and
    output paths are for variant builds such as the autotuner's."""
    os.makedirs(build_dir, exist_ok=True)
    os.makedirs(os.path.dirname(lib), exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(len(srcs), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, build_dir, tuple(defines)), srcs))
    if os.path.isfile(lib) and all(os.path.getmtime(o) <= os.path.getmtime(lib) for o in objs):
        return lib
    tmp = lib + ".tmp"
    cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
