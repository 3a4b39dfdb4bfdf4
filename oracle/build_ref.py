#!/usr/bin/env python3
"""Recipe that compiles the reference's own C sources into oracle/_ref/<config>/libref.so.

Test infrastructure only.  The reference (phynadia/Ternary-CHNS) is plain C99
whose only external dependencies are MPI and FFTW3-MPI (Makefile:1-2).  Neither
is installed here, so the build links the reference files, where they lie, against
oracle/shim/ (a single-rank MPI and an FFTW-MPI stand-in running the oracle's own
FP64 FFT, oracle/fft_cpu.c) and the harness oracle/ref_harness.c.

Every parameter of the reference is a compile-time #define in global.h/macro.h
(global.h:19-45,102-143; macro.h:1-15).  For each configuration this recipe writes
a generated global.h (the reference's file with the parameter values substituted)
and a generated macro.h into the configuration's build folder under oracle/_ref/,
and compiles with ``-I <that folder> -I-`` so that the reference's
``#include "global.h"`` resolves to the generated header instead of the file next
to the source.  Nothing in the reference's folder is written, and no reference source
is kept in the repository: oracle/_ref/ is git-ignored build output.

The reference's source folder comes only from the caller: the environment
variable CHNS_REFERENCE_DIR, set_reference_dir(), or ``--ref DIR`` on the command
line.  With none of them set, nothing is built (and the command line fails with a
message saying so).

Usage:  python oracle/build_ref.py --ref DIR [config ...]   (default: all configurations)
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("CHNS_REFERENCE_DIR") or None


def set_reference_dir(path: str | None) -> None:
    """Names the folder holding the reference's sources (global.h, etd2rk.c, ...)."""
    global REF
    REF = path or None


def _ref(*parts: str) -> str:
    if not REF:
        raise RuntimeError("the reference's source folder is not set: CHNS_REFERENCE_DIR, "
                           "set_reference_dir() or --ref DIR")
    return os.path.join(REF, *parts)
OUT = os.path.join(HERE, "_ref")

# The reference files that the hot path and its set-up/diagnostics need
# (main.c, perimeter.c, spectrum.c, write_array.c, read_array.c, forcing.c are
# not linked: the harness replaces main.c's set-up, see ref_harness.c).
REF_SOURCES = [
    "global.c", "etd2rk.c", "nonlin.c", "surface_tension.c", "chem_potential.c",
    "velocity.c", "curl.c", "functions.c", "fft.c", "init.c", "free_energy.c",
    "kinetic_energy.c", "spectrum.c", "perimeter.c",
]

# Configurations: model 0 = pure Navier-Stokes, 1 = BINARY, 2 = TERNARY.
# Values are C expressions in the reference's own macro vocabulary.
_BIN = dict(model=1, lx="(2.0*pi)", dt="(1e-3)", nu="(0.01)", lam="(0.005)", sigma="(0.2)", eps="(2.0*dx)")
_TER = dict(model=2, lx="(2.0*pi)", dt="(5e-4)", nu="(0.01)", lam="(0.005)", eps="(2.0*dx)",
            s12="(0.2)", s13="(0.3)", s23="(0.25)", xlam="(2.0)")
# The reference's own default parameters (global.h:30-31,102-104,127-133) on a small grid:
# L = 4 pi gives non-integer wavenumbers, which exercises the truncation boundary.
_BIN_DEF = dict(model=1, lx="(4.0*pi)", dt="(1e-4)", nu="(0.01)", lam="1e-6", sigma="2.0", eps="(3.0*dx)")
_TER_DEF = dict(model=2, lx="(4.0*pi)", dt="(1e-4)", nu="(0.01)", lam="(1e-4)", eps="(3.0*dx)",
                s12="(0.2)", s13="(0.2)", s23="(0.45)", xlam="(2.0)")
CONFIGS = {
    "ns32": dict(model=0, n=32, lx="(2.0*pi)", dt="(1e-3)", nu="(0.01)"),
    "bin32": dict(_BIN, n=32),
    "bin64": dict(_BIN, n=64),
    "ter32": dict(_TER, n=32),
    "ter64": dict(_TER, n=64),
    "bindef64": dict(_BIN_DEF, n=64),
    "terdef64": dict(_TER_DEF, n=64),
    # binary spinodal run, 256^2, L = 2 pi, dt = 1e-3 (1000 steps)
    "bin256": dict(_BIN, n=256),
    # ternary spinodal run, 512^2 (2000 steps).  dt = 5e-4 diverges in the
    # reference (NaN by step 5: the explicit chemical-potential term is unstable);
    # dt = 5e-5 is the largest tested value that runs the 2000 steps
    "ter512": dict(_TER, n=512, dt="(5e-5)"),
    # binary 4096^2 with the 4096^2 configuration's parameters (the reference has
    # no working forcing, so this is the unforced step; same cost per step)
    "bin4096": dict(model=1, n=4096, lx="(2.0*pi)", dt="(2e-6)", nu="(1e-3)", lam="(1e-3)",
                    sigma="(0.1)", eps="(2.0*dx)"),
    # ternary at 1024^2 for a few-step parity check of the large-grid kernels
    "ter1024": dict(_TER, n=1024, dt="(5e-6)"),
    # Taylor-Green initial vorticity (TG_INIT, init.c:38-65): pure NS at L = 2 pi, and
    # binary with the reference defaults (L = 4 pi, eps = 3 dx), whose init also lays the drop
    "nstg32": dict(model=0, n=32, lx="(2.0*pi)", dt="(1e-3)", nu="(0.01)", init="tg"),
    "bintg64": dict(_BIN_DEF, n=64, init="tg"),
    # the k-space shell initial vorticity (neither TG_INIT nor ZERO_INIT, init.c:102-182):
    # pure NS at L = 2 pi, and binary with the reference defaults (L = 4 pi, whose
    # half-integer wavenumbers put some |k| exactly half-way between two shells)
    "nssh32": dict(model=0, n=32, lx="(2.0*pi)", dt="(1e-3)", nu="(0.01)", init="shell"),
    "binsh64": dict(_BIN_DEF, n=64, init="shell"),
    # SMOOTH_FILTER (macro.h:15, functions.c:69-72): the smooth filter in place of the sharp cut
    "nssf32": dict(model=0, n=32, lx="(2.0*pi)", dt="(1e-3)", nu="(0.01)", filter=True),
    "binsf64": dict(_BIN, n=64, filter=True),
    "tersf64": dict(_TER, n=64, filter=True),
    "binsfdef64": dict(_BIN_DEF, n=64, filter=True),
}

_SUBST = {  # macro name -> key in the config dict
    "lx": "lx", "ly": "lx", "Nx": "n", "Ny": "n", "nu": "nu", "dt": "dt",
    "sigma": "sigma", "epsilon": "eps", "lambda": "lam",
    "sigma_12": "s12", "sigma_13": "s13", "sigma_23": "s23", "Xlambda": "xlam",
}


def _gen_global_h(cfg: dict) -> str:
    src = open(_ref("global.h")).read()
    out = []
    for line in src.splitlines():
        m = re.match(r"^(\s*)#define\s+(\w+)\b(.*)$", line)
        if m and m.group(2) in _SUBST and _SUBST[m.group(2)] in cfg:
            val = cfg[_SUBST[m.group(2)]]
            line = f"{m.group(1)}#define {m.group(2)} ({val})"
        out.append(line)
    return "\n".join(out) + "\n"


def _gen_macro_h(cfg: dict) -> str:
    init = cfg.get("init")
    lines = ["/* generated by oracle/build_ref.py */"]
    if init == "tg":
        lines.append("#define TG_INIT")
    elif init != "shell":  # "shell": neither macro, init.c's k-space branch
        lines.append("#define ZERO_INIT")
    if cfg.get("filter"):
        lines.append("#define SMOOTH_FILTER")
    if cfg["model"] == 1:
        lines.append("#define BINARY")
    elif cfg["model"] == 2:
        lines.append("#define TERNARY")
    return "\n".join(lines) + "\n"


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def reference_present() -> bool:
    return bool(REF) and all(os.path.isfile(os.path.join(REF, f)) for f in REF_SOURCES + ["global.h"])


def lib_path(name: str, dropin: bool = False) -> str:
    return os.path.join(OUT, name + ("_dropin" if dropin else ""), "libref.so")


def build(name: str, force: bool = False, dropin: bool = False) -> str:
    """dropin=True links ternary-chns_b200/csrc/etd2rk_dropin.c (the GPU step behind
    the reference's own etd2rk signature) in place of the reference's etd2rk.c."""
    cfg = CONFIGS[name]
    bdir = os.path.join(OUT, name + ("_dropin" if dropin else ""))
    lib = lib_path(name, dropin)
    repo = os.path.dirname(HERE)
    chns_lib_dir = os.path.join(repo, "ternary-chns_b200", "lib")
    if dropin and not os.path.isfile(os.path.join(chns_lib_dir, "libchns_b200.so")):
        raise FileNotFoundError("build libchns_b200.so before the drop-in oracle")
    deps = [os.path.join(HERE, f) for f in ("ref_harness.c", "fft_cpu.c", "fft_cpu.h", "build_ref.py",
                                            "shim/shim.c", "shim/mpi.h", "shim/fftw3-mpi.h")]
    deps += [_ref(f) for f in REF_SOURCES + ["global.h"]]
    if dropin:
        deps += [os.path.join(repo, "ternary-chns_b200", "csrc", "etd2rk_dropin.c"),
                 os.path.join(repo, "include", "chns.h"), os.path.join(chns_lib_dir, "libchns_b200.so")]
    if not force and os.path.isfile(lib):
        t = os.path.getmtime(lib)
        if all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d)):
            return lib
    os.makedirs(bdir, exist_ok=True)
    with open(os.path.join(bdir, "global.h"), "w") as f:
        f.write(_gen_global_h(cfg))
    with open(os.path.join(bdir, "macro.h"), "w") as f:
        f.write(_gen_macro_h(cfg))
    cc = os.environ.get("CC", "gcc")
    flags = ["-O2", "-ffp-contract=off", "-fPIC", "-w", "-fvisibility=hidden", "-std=gnu99"]
    inc = ["-I", bdir, "-I-", "-I", os.path.join(HERE, "shim")]
    objs = []
    # free_energy.c only compiles with a phase field (it prints to `fe`, which
    # global.h declares under BINARY/TERNARY only)
    sources = [s for s in REF_SOURCES if cfg["model"] != 0 or s != "free_energy.c"]
    if dropin:
        sources = [s for s in sources if s != "etd2rk.c"]
    for s in sources:
        o = os.path.join(bdir, s.replace(".c", ".o"))
        _run([cc, *flags, *inc, "-c", _ref(s), "-o", o])
        objs.append(o)
    if dropin:
        o = os.path.join(bdir, "etd2rk_dropin.o")
        _run([cc, *flags, *inc, "-I", os.path.join(repo, "include"), "-c",
              os.path.join(repo, "ternary-chns_b200", "csrc", "etd2rk_dropin.c"), "-o", o])
        objs.append(o)
    for s in ("ref_harness.c",):
        o = os.path.join(bdir, s.replace(".c", ".o"))
        _run([cc, *flags, *inc, "-c", os.path.join(HERE, s), "-o", o])
        objs.append(o)
    for s in ("shim/shim.c", "fft_cpu.c"):
        o = os.path.join(bdir, os.path.basename(s).replace(".c", ".o"))
        _run([cc, *flags, "-I", os.path.join(HERE, "shim"), "-c", os.path.join(HERE, s), "-o", o])
        objs.append(o)
    tmp = lib + ".tmp"
    link = ["-lm", "-lpthread"]
    if dropin:
        rel = os.path.relpath(chns_lib_dir, bdir)
        link = ["-L", chns_lib_dir, "-lchns_b200", f"-Wl,-rpath,$ORIGIN/{rel}"] + link
    _run([cc, "-shared", "-Wl,-Bsymbolic", "-o", tmp, *objs, *link])
    os.replace(tmp, lib)
    for o in objs:
        os.remove(o)
    return lib


# configurations also built with the drop-in etd2rk (needs libchns_b200.so)
DROPIN_CONFIGS = ["ns32", "bin32", "ter32", "bindef64", "terdef64", "binsf64"]


def build_all(names=None, force=False, dropin: bool = True) -> list[str]:
    if not reference_present():
        return []
    out = [build(n, force) for n in (names or list(CONFIGS))]
    if dropin:
        for n in DROPIN_CONFIGS:
            if names is None or n in names:
                out.append(build(n, force, dropin=True))
    return out


if __name__ == "__main__":
    args = sys.argv[1:]
    if "--ref" in args:
        k = args.index("--ref")
        set_reference_dir(args[k + 1])
        del args[k:k + 2]
    names = args or None
    if not REF:
        sys.exit("build_ref.py: give the reference's source folder with --ref DIR or CHNS_REFERENCE_DIR")
    if not reference_present():
        sys.exit(f"build_ref.py: the reference's sources are not under {REF}")
    for p in build_all(names, force=True):
        print(p)
