#!/usr/bin/env python3
"""Benchmark of the ETD2RK CHNS step on B200 (one JSON line on rank 0).

Workload: binary CHNS on a 4096^2 grid (the configuration the metric is quoted
on): Kolmogorov forcing F0 sin(4y) x-hat, F0 = 1, nu = M = 1e-3, sigma = 0.1,
eps = 2 dx, 64 tanh drops of radius 0.3 on c = 0 and random vorticity modes
|k| <= 8 at rms 0.1, all seeded synthetic inputs.  Headline precision
CHNS_FP32_STATE64: FP32 transforms and pointwise arithmetic, ETD coefficients
from FP64 (series for small |c h|), the state carried as float pairs (hi + lo)
inside the truncation disc with the ETD update in FP64, k = 0 modes in FP64 --
the FP32 mode whose state stays within 1e-5 relative L2 of the FP64 step after
1000 steps (`--precision fp32` times the plain FP32 state instead; the other mode
is reported beside it).  A "step" is one full ETD2RK step (both stages).

  value    : steps/s of the whole job (all ranks), state resident in HBM
  e2e      : steps/s through the reference-facing call with HOST buffers: every
             step uploads the FFTW-layout state from pinned memory, steps once and
             reads it back (the contract of the drop-in etd2rk())
  roofline : the dominant kernel's algorithmic bytes / its CUDA-event time
  cpu_baseline : the reference's own etd2rk() (compiled here, oracle/_ref)
             timed on the host cores on a sample of the same workload
  adjoint  : the discrete adjoint (chns_adjoint) of 200 binary steps at 512^2
             (nu = 0.01, M = 0.005, sigma = 0.2, eps = 2 dx, spinodal noise;
             dt = 1e-4: with eps = 2 dx the explicit bulk term grows as n^3 and
             dt = 1e-3 diverges at 512^2), checkpoints every 20 steps: its time
             over the forward time of the same 200 steps, in FP64 and FP32,
             central differences along seeded directions, and a 4096^2 run of
             1000 steps (dt = 1.5e-7 for the same reason) for the memory budget
  diagnostics / init : per-step diagnostics (free and kinetic energy, spectra,
             perimeter) and init.c's initial conditions on the device at 4096^2,
             beside the reference's own diagnostics on the host cores
  ensemble : 64 ternary runs (32 at 256^2, 24 at 512^2, 8 at 1024^2; own seeds
             and sigma_ij ~ U[0.15, 0.35] with every gamma_i >= 0.1; nu = 0.01,
             M = 0.005, eps = 2 dx; FP32)
             advanced together by chns_ensemble_step against the same members
             stepped one after another (wall clock with a synchronize on both
             sides; dt per size so that every run stays finite)

--impl reference times the reference's CPU implementation (oracle/_ref) on the
same metric; multi-GPU runs are independent replicas (the step does not shard;
one all-to-all per transform would be the only way to split a field).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ternary-chns_b200"))

N_DEFAULT = 4096
# The headline precision is CHNS_FP32_STATE64: the FP32 right-hand side with the
# state carried as a float pair, the FP32 mode that stays within 1e-5 relative L2
# of the FP64 step after 1000 steps (the plain FP32 state drifts to ~1e-4).
METRIC = "steps/s @4096^2 binary CHNS ETD2RK, FP32 within 1e-5 rel L2 of FP64 (FP32_STATE64)"
METRIC_PLAIN = "steps/s @4096^2 binary CHNS ETD2RK (plain FP32 state, FP64 coefficients)"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# dt of the 4096^2 workload: the specified 2e-4 diverges under the reference's
# scheme at this resolution (the explicit bulk term exceeds the exactly
# integrated k^4 term near the truncation radius); 2e-6 runs stably.  The cost
# of a step does not depend on dt.
DT_DEFAULT = 2e-6


PREC_NOTE = {
    1: "FP32 transforms and point-wise work; ETD coefficients from FP64; k = 0 modes in FP64; FP32 state",
    2: "CHNS_FP32_STATE64: the FP32 right-hand side; w and c carried as float pairs (hi + lo) inside the "
       "truncation disc, the ETD update in float-float arithmetic (e - 1 from expm1); k = 0 modes in FP64",
}


def workload_params(n: int, precision: int, coef_mode: int = 1, dt: float = DT_DEFAULT) -> dict:
    from chns_b200 import configs

    return configs.binary(n, dt, 1e-3, 1e-3, 0.1, precision, coef_mode, force_amp=1.0, force_k=4.0)


def initial_fields(n: int):
    from chns_b200 import configs

    _, c0, w0 = configs.binary_kolmogorov(n)
    return c0, w0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[3 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def read_profile_value(kernel: str, n: int, key: str):
    """A figure of the committed ncu summary profiles/<kernel>_<n>_fp32.md (a line
    '<key>: <number>'), or None."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{n}_fp32.md")
    try:
        for line in open(path):
            if line.strip().startswith(key + ":"):
                v = float(line.split(":", 1)[1].strip())
                return int(v) if v.is_integer() else v
    except (OSError, ValueError):
        pass
    return None


def read_profile_traffic(kernel: str, n: int):
    """DRAM bytes per launch of `kernel` from the committed ncu summary
    profiles/<kernel>_<n>_fp32.md (a line 'dram_bytes_per_launch: <int>')."""
    return read_profile_value(kernel, n, "dram_bytes_per_launch")


def init_leg(C, n: int) -> dict:
    """Wall time of init.c's initial conditions on the device at n^2 (each call
    ends with a synchronize): binary drop, Taylor-Green vorticity, ternary noise
    (host draws of the C library generator + device fields and transforms)."""
    out = {"grid": n, "precision": "fp32"}
    lx = 2 * math.pi
    for model, key in ((1, "binary"), (2, "ternary")):
        p = dict(model=model, precision=1, nx=n, ny=n, lx=lx, ly=lx, dt=1e-6, nu=0.01, epsilon=2 * lx / n,
                 sigma=0.2, sigma12=0.2, sigma13=0.3, sigma23=0.25)
        p["lambda"] = 0.005
        with C.Context(p) as c:
            c.init_vorticity(C.INIT_W_TAYLOR_GREEN, 1.0)  # first call: buffers and kernels warm
            t0 = time.perf_counter()
            c.init_vorticity(C.INIT_W_TAYLOR_GREEN, 1.0)
            t1 = time.perf_counter()
            c.init_phase(C.INIT_C_DROP if model == 1 else C.INIT_C_NOISE, 10)
            t2 = time.perf_counter()
        if model == 1:
            out["taylor_green_ms"] = round((t1 - t0) * 1e3, 3)
            out["drop_ms"] = round((t2 - t1) * 1e3, 3)
        else:
            out["ternary_noise_ms"] = round((t2 - t1) * 1e3, 3)
    return out


def diagnostics_leg(C, n: int, st0, cpu: bool) -> dict:
    """Wall time (each call ends with a synchronize) of the per-step diagnostics at
    n^2 on the bench state: free and kinetic energy (chns_diagnostics), spectra
    (chns_spectrum), perimeter (chns_perimeter), FP32 and FP64 contexts; with
    cpu=True also the reference's own free_energy(), kinetic_energy(), spectrum()
    and perimeter() (oracle/_ref/bin<n>, oracle FFT on all host threads)."""
    import tempfile

    out = {"grid": n}
    for prec, key in ((C.FP32, "gpu_fp32_ms"), (C.FP64, "gpu_fp64_ms")):
        with C.Context(workload_params(n, prec)) as c:
            c.set_state(*st0)
            c.diagnostics(), c.spectrum(), c.perimeter()  # warm
            t = {}
            for nm, fn in (("energies", c.diagnostics), ("spectrum", c.spectrum), ("perimeter", c.perimeter)):
                t0 = time.perf_counter()
                fn()
                t[nm] = round((time.perf_counter() - t0) * 1e3, 3)
            out[key] = t
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        name = f"bin{n}"
        if os.path.isfile(O.build_ref.lib_path(name)):
            thr = os.cpu_count() or 1
            R = O.RefLib(name, nthreads=thr)
            R.set_state(*st0)
            t = {}
            work = tempfile.mkdtemp()
            for nm, fn in (("free_energy", R.free_energy), ("kinetic_energy", R.kinetic_energy),
                           ("spectrum", lambda: R.spectrum(work)), ("perimeter", R.perimeter)):
                t0 = time.perf_counter()
                fn()
                t[nm] = round((time.perf_counter() - t0) * 1e3, 1)
            out["reference_cpu_ms"] = t
            out["reference_cores"] = thr
    return out


def replica_throughput(ms: float, steps: int, world: int, device: str):
    """Whole-job steps/s of `world` independent replicas (one per rank and GPU, no
    data-path collective): every rank ran `steps` steps in `ms` milliseconds; the
    job takes as long as its slowest rank.  Returns (max ms over ranks, steps/s)."""
    t_max = ms
    if world > 1:
        import torch
        import torch.distributed as dist

        t = torch.tensor([ms], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    return t_max, world * steps / (t_max / 1e3)


def adjoint_params(n: int, precision: int, dt: float) -> dict:
    from chns_b200 import configs

    return configs.binary_adjoint(n, precision, dt)[0]


def adjoint_leg(C, stream, big_steps: int):
    """Cost of the discrete adjoint against the forward steps it reverses."""
    import numpy as np
    import torch

    from chns_b200 import configs

    n, steps, ckpt = 512, 200, 20
    c_real = configs.binary_adjoint(n)[1]
    out = {"grid": n, "steps": steps, "ckpt": ckpt, "loss": "E_bulk + E_grad + <|grad phi|^2> at the final step",
           "timing": "median of 3 CUDA-event timings each"}
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    def timed_pair(c, st0):
        """Median of 3 CUDA-event timings of `steps` forward steps and of the adjoint
        of the same steps from st0 (after one untimed adjoint: buffers, graph)."""
        c.adjoint(steps, ckpt)
        c.step(10)
        tf, ta = [], []
        for _ in range(3):
            c.set_state(*st0)
            c.synchronize()
            ev0.record(stream)
            c.step(steps)
            ev1.record(stream)
            ev1.synchronize()
            tf.append(ev0.elapsed_time(ev1))
        for _ in range(3):
            c.set_state(*st0)
            c.synchronize()
            ev0.record(stream)
            res = c.adjoint(steps, ckpt)
            ev1.record(stream)
            ev1.synchronize()
            ta.append(ev0.elapsed_time(ev1))
        return statistics.median(tf), statistics.median(ta), res

    for prec, name in ((C.FP64, "fp64"), (C.FP32, "fp32")):
        with C.Context(adjoint_params(n, prec, 1e-4)) as c:
            c.L.chns_set_stream(c.handle, ctypes_stream(stream))
            c.set_phase_real(c_real)
            st0 = c.get_state()
            t_fwd, t_adj, (J, gw, gc, gp) = timed_pair(c, st0)
            leg = {"forward_ms": round(t_fwd, 3), "adjoint_ms": round(t_adj, 3), "ratio": round(t_adj / t_fwd, 3),
                   "J": J, "dJ_dnu": gp[0], "dJ_dM": gp[1], "dJ_dsigma": gp[2]}
            if prec == C.FP64:
                # central differences of J along seeded smooth directions of c_hat_0, at
                # h = 1e-6 and 1e-5 (J ~ 1.6e3: the rounding of J limits h = 1e-6 to
                # ~eps J / (h |dJ|) relative; the O(h^2) error of 1e-5 is ~1e-10)
                fds = []
                mx = np.minimum(np.arange(n), n - np.arange(n))
                kk = np.sqrt(mx[:, None] ** 2 + np.arange(n // 2 + 1)[None, :] ** 2)
                for k in range(2):
                    d = np.fft.rfft2(np.random.default_rng(100 + k).standard_normal((n, n)))
                    d *= np.exp(-kk / 8.0)
                    d *= np.abs(st0[1]).ravel()[1:].max() / np.abs(d).max()
                    d[0, 0] = 0.0
                    ad = float(np.sum(gc.real * d.real + gc.imag * d.imag))
                    row = {"adjoint": ad}
                    for h in (1e-6, 1e-5):
                        js = []
                        for sgn in (1, -1):
                            c.set_state(st0[0], st0[1] + sgn * h * d)
                            js.append(c.adjoint(steps, ckpt)[0])
                        fd = (js[0] - js[1]) / (2 * h)
                        row[f"rel_err_h{h:g}"] = abs(ad - fd) / abs(fd)
                    fds.append(row)
                leg["fd"] = fds
                g64 = (gc, gp)
            else:
                leg["rel_diff_vs_fp64_dJ_dc"] = float(np.linalg.norm(gc - g64[0]) / np.linalg.norm(g64[0]))
            out[name] = leg
    # ternary: the spinodal setting at 512^2 (dt = 5e-5), same schedule
    from chns_b200 import configs as _cf

    pt, ph = _cf.ternary_spinodal(n, C.FP64)
    for prec, name in ((C.FP64, "ternary_fp64"), (C.FP32, "ternary_fp32")):
        with C.Context(dict(pt, precision=prec)) as c:
            c.L.chns_set_stream(c.handle, ctypes_stream(stream))
            c.set_phase_real(*ph)
            st0 = c.get_state()
            t_fwd, t_adj, (J, _, _, gp) = timed_pair(c, st0)
            out[name] = {"forward_ms": round(t_fwd, 3), "adjoint_ms": round(t_adj, 3),
                         "ratio": round(t_adj / t_fwd, 3), "J": J,
                         "dJ_dparams": dict(zip(("nu", "M", "sigma12", "sigma13", "sigma23"), map(float, gp)))}
    if big_steps > 0:
        nb = 4096
        with C.Context(adjoint_params(nb, C.FP32, 1.5e-7)) as c:
            c.L.chns_set_stream(c.handle, ctypes_stream(stream))
            noise = np.random.default_rng(7).uniform(-0.05, 0.05, (nb, nb))
            c.set_phase_real(0.5 * (1.0 + noise - noise.mean()))
            st_big = c.get_state()
            c.step(3)
            c.set_state(*st_big)
            c.synchronize()
            ev0.record(stream)
            c.step(big_steps)
            ev1.record(stream)
            ev1.synchronize()
            t_fwd = ev0.elapsed_time(ev1) / 1e3
            c.set_state(*st_big)
            c.synchronize()
            free0, total = torch.cuda.mem_get_info()
            ev0.record(stream)
            J = c.adjoint(big_steps, ckpt)[0]
            ev1.record(stream)
            ev1.synchronize()
            free1, _ = torch.cuda.mem_get_info()
            t_adj = ev0.elapsed_time(ev1) / 1e3
            out["fp32_4096"] = {"steps": big_steps, "ckpt": ckpt, "forward_s": round(t_fwd, 3),
                                "adjoint_s": round(t_adj, 3), "ratio": round(t_adj / t_fwd, 3),
                                "adjoint_buffers_gb": round((free0 - free1) / 1e9, 2),
                                "hbm_total_gb": round(total / 1e9, 1), "J_finite": bool(math.isfinite(J))}
    return out


def ensemble_members(seed: int = 3000):
    from chns_b200 import configs

    return configs.ternary_ensemble(seed)


def ternary_leg(C, stream, n: int = 4096, steps: int = 100) -> dict:
    """The ternary model at n^2 (sigma_12/13/23 = 0.2/0.3/0.25, nu = 0.01, M = 0.005,
    eps = 2 dx, dt = 5e-8: stable at this resolution; spinodal noise c_i = 1/3 +
    U[-0.02, 0.02]): steps/s per precision (CUDA events on the context's stream), and
    the relative L2 distance of the FP32 states from the FP64 one after `steps`."""
    import numpy as np

    from chns_b200 import configs

    p = configs.ternary(n, 5e-8, 0.01, 0.005, 0.2, 0.3, 0.25, coef_mode=1)
    rng = np.random.default_rng(7)
    ph = (1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n)), 1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n)))
    import torch

    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    out, states = {"grid": n, "steps": steps, "dt": 5e-8}, {}
    for prec, name in ((C.FP64, "fp64"), (C.FP32, "fp32"), (C.FP32_STATE64, "fp32_state64")):
        with C.Context(dict(p, precision=prec)) as c:
            c.set_phase_real(*ph)
            C.load_library().chns_set_stream(c.handle, ctypes_stream(stream))
            c.step(3)
            c.synchronize()
            ev0.record(stream)
            c.step(steps)
            ev1.record(stream)
            ev1.synchronize()
            out[f"{name}_steps_per_s"] = round(steps / (ev0.elapsed_time(ev1) / 1e3), 2)
            states[name] = c.get_state()
    for name in ("fp32", "fp32_state64"):
        out[f"{name}_rel_l2_vs_fp64"] = [float(np.linalg.norm(b - a) / np.linalg.norm(a))
                                         for a, b in zip(states["fp64"], states[name])]
    return out


def ensemble_leg(C, steps: int):
    """Throughput of the 64-member ternary ensemble, together and one by one."""
    import numpy as np
    from chns_b200.configs import ENSEMBLE_GROUPS

    members = ensemble_members()
    pts = sum(p["nx"] * p["ny"] for p, _ in members)
    times, launches, finite = {}, {}, None
    with C.Ensemble([p for p, _ in members]) as ens:
        try:
            ens.persistent = True
            persistent = True
        except C.ChnsError:
            persistent = False
        # the graph of per-member branches, then (when the members allow it) the
        # persistent kernel, each from the same initial state
        for mode in ([False, True] if persistent else [False]):
            ens.persistent = mode
            for m, (_, ph) in zip(ens.members, members):
                m.set_phase_real(*ph)
            ens.step(5)
            ens.synchronize()
            t0 = time.perf_counter()
            ens.step(steps)
            ens.synchronize()
            times[mode] = time.perf_counter() - t0
            # persistent: one cooperative launch (and a memset of its barrier counters) per step
            launches[mode] = steps if mode else sum(m.launches_per_step() for m in ens.members) * steps
            fin = [bool(np.all(np.isfinite(m.get_state()[1]))) for m in ens.members]
            f = {f"{n}^2": all(f for f, (p, _) in zip(fin, members) if p["nx"] == n) for n, _, _ in ENSEMBLE_GROUPS}
            finite = f if finite is None else {k: finite[k] and f[k] for k in f}
    best = True if persistent and times[True] <= times[False] else False
    t_ens = times[best]
    t_one = 0.0
    for p, ph in members:
        with C.Context(p) as c:
            c.set_phase_real(*ph)
            c.step(5)
            c.synchronize()
            t0 = time.perf_counter()
            c.step(steps)
            c.synchronize()
            t_one += time.perf_counter() - t0
    return {"members": {f"{n}^2": k for n, k, _ in ENSEMBLE_GROUPS}, "model": "ternary", "precision": "fp32",
            "steps": steps, "ensemble_s": round(t_ens, 4), "one_by_one_s": round(t_one, 4),
            "speedup": round(t_one / t_ens, 3), "member_steps_per_s": round(len(members) * steps / t_ens, 1),
            "grid_point_steps_per_s": round(pts * steps / t_ens, 1), "gpu_launches": launches[best],
            "mode": "persistent kernel" if best else "graph of per-member branches",
            "persistent_s": round(times[True], 4) if persistent else None, "graph_s": round(times[False], 4),
            "all_finite": finite}


def run_gpu(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    import chns_b200 as C

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    n = args.n
    L = C.load_library()

    def barrier():
        if world > 1:
            dist.barrier()

    # the initial spectral state, built once in FP64 (init.c INIT_READ_DATA path)
    c0, w0 = initial_fields(n)
    with C.Context(workload_params(n, C.FP64, dt=args.dt)) as cinit:
        cinit.set_phase_real(c0)
        st0 = cinit.get_state()
    st0[0] = w0
    del c0

    # ---------------- device-resident throughput (headline precision) ----------------
    main_prec = C.FP32_STATE64 if args.precision == "fp32_state64" else C.FP32
    other_prec = C.FP32 if main_prec == C.FP32_STATE64 else C.FP32_STATE64
    ctx = C.Context(workload_params(n, main_prec, dt=args.dt))
    ctx.set_state(*st0)
    stream = torch.cuda.Stream()
    L.chns_set_stream(ctx.handle, ctypes_stream(stream))
    ctx.step(args.warmup)
    ctx.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        time.sleep(0.3)  # let nvidia-smi start sampling before the timed region
        ev0.record(stream)
        ctx.step(args.steps)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    t_max, value = replica_throughput(ms, args.steps, world, "cuda")
    ms_per_step = t_max / args.steps
    launches = ctx.launches_per_step() * args.steps
    fe, ke, rc = ctx.diagnostics()
    finite = rc == 0

    # ---------------- per-kernel times of one step (events between launches) ----------------
    prof = profile_kernels(ctx, L, stream, reps=max(3, min(10, args.steps)))

    # ---------------- end to end through the host-buffer call ----------------
    e2e = e2e_host_loop(ctx, stream, max(3, min(args.steps, 10)))
    ctx.close()

    # ---------------- the other FP32 mode on the same workload ----------------
    other = None
    if args.other_steps > 0:
        cs = C.Context(workload_params(n, other_prec, dt=args.dt))
        cs.set_state(*st0)
        L.chns_set_stream(cs.handle, ctypes_stream(stream))
        cs.step(3)
        cs.synchronize()
        ev0.record(stream)
        cs.step(args.other_steps)
        ev1.record(stream)
        ev1.synchronize()
        o_sps = args.other_steps / (ev0.elapsed_time(ev1) / 1e3)
        o_prof = profile_kernels(cs, L, stream, reps=5)
        cs.close()
        other = {"steps_per_s": round(o_sps, 3), "steps": args.other_steps, "per_kernel_ms": o_prof["per_kernel_ms"],
                 "note": PREC_NOTE[other_prec]}

    # ---------------- FP64 plain step (reference coefficients) on the same workload ----------------
    ctx64 = C.Context(workload_params(n, C.FP64, coef_mode=0, dt=args.dt))
    ctx64.set_state(*st0)
    L.chns_set_stream(ctx64.handle, ctypes_stream(stream))
    ctx64.step(3)
    ctx64.synchronize()
    k64 = max(5, args.steps // 4)
    ev0.record(stream)
    ctx64.step(k64)
    ev1.record(stream)
    ev1.synchronize()
    fp64_sps = k64 / (ev0.elapsed_time(ev1) / 1e3)
    ctx64.close()

    # ---------------- FP32 against FP64 after the same number of steps ----------------
    acc = None
    if args.accuracy_steps > 0:
        res = []
        for prec in (C.FP64, C.FP32, C.FP32_STATE64):
            with C.Context(workload_params(n, prec, coef_mode=1, dt=args.dt)) as c:
                c.set_state(*st0)
                c.step(args.accuracy_steps)
                res.append(c.get_state())
        err = [float(np.linalg.norm(b - a) / np.linalg.norm(a)) for a, b in zip(res[0], res[1])]
        err64 = [float(np.linalg.norm(b - a) / np.linalg.norm(a)) for a, b in zip(res[0], res[2])]
        drift = [float(abs(r[1][0, 0] - st0[1][0, 0]) / abs(st0[1][0, 0])) for r in res[1:]]
        acc = {"steps": args.accuracy_steps, "reference": "FP64 step, same coefficients (series/expm1)",
               "fp32_state64": {"rel_l2_w": err64[0], "rel_l2_c": err64[1], "mean_c_rel_drift": drift[1],
                                "within_1e-5": max(err64) <= 1e-5},
               "fp32_plain": {"rel_l2_w": err[0], "rel_l2_c": err[1], "mean_c_rel_drift": drift[0],
                              "within_1e-5": max(err) <= 1e-5}}
        del res

    # single-GPU legs (the other ranks of a replica run would only wait for them)
    solo = world == 1
    init = init_leg(C, n) if solo else None
    diag = diagnostics_leg(C, n, st0, not args.no_cpu_baseline) if solo else None
    adj = adjoint_leg(C, stream, args.adjoint_big_steps) if args.adjoint and solo else None
    ens = ensemble_leg(C, args.ensemble_steps) if args.ensemble_steps > 0 and solo else None
    tern = ternary_leg(C, stream, n) if args.ternary and solo else None

    out = None
    if rank == 0:
        hbm, src = peaks()
        dom = max(prof["per_kernel_ms"].items(), key=lambda kv: kv[1]) if prof["per_kernel_ms"] else (None, None)
        kb = prof["bytes"]
        roof = None
        if dom[0]:
            ach = kb[dom[0]] / (dom[1] / 1e3) / 1e9
            roof = {"kernel": dom[0], "bound": "hbm", "achieved": round(ach, 1), "peak": hbm, "peak_source": src,
                    "unit": "GB/s", "frac": round(ach / hbm, 4), "traffic": read_profile_traffic(dom[0], n),
                    "algorithmic_bytes_per_launch": kb[dom[0]], "ms_per_launch": round(dom[1], 4),
                    "issue_active_pct": read_profile_value(dom[0], n, "issue_active_pct"),
                    "warps_active_pct": read_profile_value(dom[0], n, "warps_active_pct"),
                    "note": "no stage is a contraction, so the HBM roofline is the one that applies; the row "
                            "kernels reach a fraction of it because they are latency-bound (two 256-thread CTAs "
                            "per SM at 128 registers, barrier-synchronous transforms): see profiles/"}
        rsz = 4
        model_bytes = 120 * n * n * rsz
        # the bytes the fused kernels need: each of the five stage kernels runs once per stage
        fused_bytes = 2 * sum(kb.values())
        fused_gbs = fused_bytes * value / world / 1e9
        if roof is not None:
            roof["step_fused"] = {"bytes_per_step": fused_bytes, "achieved_gbs": round(fused_gbs, 1),
                                  "frac": round(fused_gbs / hbm, 4),
                                  "note": "whole step: the five stage kernels' algorithmic bytes x 2 stages / "
                                          "ms_per_step, against the same peak"}
        acc_short = None
        if acc is not None:
            acc_short = {"steps": acc["steps"],
                         "fp32_state64": [round(acc["fp32_state64"]["rel_l2_w"], 9),
                                          round(acc["fp32_state64"]["rel_l2_c"], 9)],
                         "fp32_plain": [round(acc["fp32_plain"]["rel_l2_w"], 9),
                                        round(acc["fp32_plain"]["rel_l2_c"], 9)],
                         "order": "rel L2 of (omega, c) against the FP64 step"}
        out = {
            "metric": METRIC if main_prec == C.FP32_STATE64 else METRIC_PLAIN, "value": round(value, 3),
            "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "fp64_steps_per_s": round(fp64_sps, 3),
            "fp32_over_fp64": round((value / world) / fp64_sps, 3),
            "accuracy_vs_fp64": acc_short,
            "step_fused_frac": round(fused_gbs / hbm, 4),
            "config": {"workload": f"binary CHNS {n}^2, Kolmogorov forcing F0=1 kf=4, 64 drops R=0.3, "
                                   f"nu=M=1e-3, sigma=0.1, eps=2dx, dt={args.dt:g}",
                       "grid": n, "model": "binary", "precision": PREC_NOTE[main_prec],
                       "l2": "inputs larger than L2 (state and intermediates ~1 GB); no flush needed",
                       "parallelism": f"replicas x{world}"},
            "e2e": e2e,
            "roofline": roof,
            "step_model": {"bytes_per_step": model_bytes, "achieved_gbs": round(model_bytes * value / world / 1e9, 1),
                           "frac_of_peak": round(model_bytes * value / world / 1e9 / hbm, 4),
                           "note": "whole step against the 120 N^2 s bytes/step model"},
            "grid_point_steps_per_s": round(value * n * n, 1),
            "fp32_vs_fp64": acc,
            ("fp32_plain" if main_prec == C.FP32_STATE64 else "fp32_state64"): other,
            "init": init,
            "diagnostics": diag,
            "adjoint": adj,
            "ensemble": ens,
            "ternary": tern,
            "per_kernel_ms": prof["per_kernel_ms"],
            "gpu_launches": launches,
            "state_finite": bool(finite),
            "clocks": clk.summary(),
        }
        if not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(n, args.cpu_steps)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if out:
        print(json.dumps(out))


def run_profile_case(args):
    """A small, fixed piece of work for an ncu capture: "step" = the workload's FP32
    context stepped --steps times ("step_state64": the CHNS_FP32_STATE64 context); "adjoint" = one adjoint of --steps steps (K = 20)
    at 512^2 FP64 after a warm-up call; "adjoint_2048" = one binary adjoint of --steps
    steps (K = 20) at 2048^2 FP32, whose fields are larger than L2; "ensemble" = --steps
    ensemble steps of the 64-member ternary ensemble."""
    import torch

    import chns_b200 as C

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if args.profile_case == "adjoint":
        from chns_b200 import configs

        p, c_real = configs.binary_adjoint(512, C.FP64)
        with C.Context(p) as c:
            c.set_phase_real(c_real)
            c.adjoint(4, 20)
            c.adjoint(args.steps, 20)
        return
    if args.profile_case == "adjoint_2048":
        from chns_b200 import configs

        p, c_real = configs.binary_adjoint(2048, C.FP32)
        with C.Context(p) as c:
            c.set_phase_real(c_real)
            c.adjoint(args.steps, 20)
        return
    if args.profile_case == "ensemble":
        members = ensemble_members()
        with C.Ensemble([p for p, _ in members]) as ens:
            for m, (_, ph) in zip(ens.members, members):
                m.set_phase_real(*ph)
            ens.step(args.steps)
            ens.synchronize()
        return
    n = args.n
    c0, w0 = initial_fields(n)
    prec = C.FP32_STATE64 if args.profile_case == "step_state64" else C.FP32
    with C.Context(workload_params(n, prec, dt=args.dt)) as ctx:
        ctx.set_phase_real(c0)
        st = ctx.get_state()
        st[0] = w0
        ctx.set_state(*st)
        ctx.step(args.steps)
        ctx.synchronize()


def ctypes_stream(stream):
    import ctypes

    return ctypes.c_void_p(stream.cuda_stream)


def profile_kernels(ctx, L, stream, reps: int):
    """Times every kernel of one step with CUDA events recorded between launches
    on the context's stream (outside the graph; same kernels, same arguments)."""
    import ctypes

    import torch

    maxk = 64
    arr = (ctypes.c_float * maxk)()
    names = (ctypes.c_int * maxk)()
    L.chns_profile_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    L.chns_profile_step.restype = ctypes.c_int
    nk = L.chns_profile_step(ctx.handle, reps, arr, names, maxk)
    kinds = {0: "spec_inv", 1: "row_adv", 2: "spec_fwd_c", 3: "row_force", 4: "spec_curl_w", 5: "row_adv_b"}
    per = {}
    cnt = {}
    for k in range(max(nk, 0)):
        nm = kinds.get(names[k], str(names[k]))
        per[nm] = per.get(nm, 0.0) + arr[k]
        cnt[nm] = cnt.get(nm, 0) + 1
    per_launch = {k: per[k] / cnt[k] for k in per}
    n = ctx.nx
    jt = n // 4
    cx = 16 if ctx.params.get("precision", 0) == 0 else 8
    S = (n // 2 + 1) * n * cx
    G = (jt + 1) * n * cx
    disc = disc_modes(n) * cx
    bytes_ = {
        "spec_inv": 2 * disc + 7 * G,
        "row_adv": 7 * G + 3 * S,
        "spec_fwd_c": 3 * S + S + S + G + S + S,
        "row_force": 3 * G + 2 * S,
        "spec_curl_w": 2 * S + S + S + S + S,
    }
    if ctx.params.get("precision", 0) == 2:
        # float-pair state: the low parts inside the truncation disc, read and written by the update
        bytes_["spec_fwd_c"] += 2 * disc
        bytes_["spec_curl_w"] += 2 * disc
    return {"per_kernel_ms": {k: round(v, 4) for k, v in per_launch.items()}, "bytes": bytes_}


def disc_modes(n: int) -> int:
    fx = 1.0
    dax = (n / 4.0) * fx
    lim2 = dax * dax
    cnt = 0
    for j in range(n // 2 + 1):
        ky = fx * j
        for m in range(n // 2 + 1):
            kx = fx * m
            if kx * kx + ky * ky > lim2:
                break
            cnt += 1 if m == 0 else 2
    return cnt


def e2e_host_loop(ctx, stream, steps: int):
    """The drop-in contract: host FFTW-layout state in, one step, state out."""
    import numpy as np
    import torch

    n = ctx.nx
    shape = (n, n // 2 + 1)
    pin = [torch.empty(shape[0] * shape[1] * 2, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    st = ctx.get_state()
    for a, s in zip(pin, st):
        a.numpy()[:] = s.view(np.float64).ravel()
    L = ctx.L
    ptrs = [a.data_ptr() for a in pin]
    import ctypes

    def ok(what, rc):
        if rc != 0:
            raise RuntimeError(f"{what} returned {rc} in the end-to-end leg")

    def one():
        ok("chns_set_state", L.chns_set_state(ctx.handle, ctypes.c_void_p(ptrs[0]), ctypes.c_void_p(ptrs[1]), None, 0))
        ok("chns_step", L.chns_step(ctx.handle, 1))
        ok("chns_get_state", L.chns_get_state(ctx.handle, ctypes.c_void_p(ptrs[0]), ctypes.c_void_p(ptrs[1]), None, 0))

    one()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    ev1.record(stream)
    ev1.synchronize()
    wall = time.perf_counter() - t0
    bytes_ = 2 * shape[0] * shape[1] * 16
    return {"value": round(steps / wall, 3), "unit": "steps/s", "h2d_bytes_per_step": bytes_,
            "d2h_bytes_per_step": bytes_, "note": "chns_set_state(host) + chns_step(1) + chns_get_state(host), page-locked host "
                    "arrays (the drop-in etd2rk() page-locks the reference's arrays with chns_pin_host)"}


def cpu_baseline(n: int, steps: int, threads: int | None = None):
    """The reference's own etd2rk() (oracle/_ref/bin<n>) on the host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    name = f"bin{n}"
    if not os.path.isfile(O.build_ref.lib_path(name)):
        return {"value": None, "unit": "steps/s", "kind": "reference", "cores": 0,
                "sample": f"oracle/_ref/{name} not built"}
    thr = threads or os.cpu_count() or 1
    R = O.RefLib(name, nthreads=thr)
    c0, _ = initial_fields(n) if n >= 256 else (None, None)
    R.set_phase_real(c0)
    R.step(1)
    t0 = time.perf_counter()
    R.step(steps)
    el = time.perf_counter() - t0
    return {"value": round(steps / el, 5), "unit": "steps/s", "kind": "reference", "cores": thr,
            "sample": f"{steps} reference etd2rk() steps at {n}^2 binary (unforced: the reference has no working "
                      f"forcing), FFTW replaced by the oracle FFT on {thr} threads, reference loops single-threaded, "
                      f"-O2"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    n = args.n
    name = f"bin{n}"
    if not os.path.isfile(O.build_ref.lib_path(name)):
        print(json.dumps({"impl": "reference", "unavailable": f"oracle/_ref/{name}/libref.so not built"}))
        return
    thr = os.cpu_count() or 1
    R = O.RefLib(name, nthreads=thr)
    c0, _ = initial_fields(n)
    R.set_phase_real(c0)
    R.step(args.warmup)
    t0 = time.perf_counter()
    R.step(args.steps)
    el = time.perf_counter() - t0
    v = args.steps / el
    sample = (f"{args.steps} reference etd2rk() steps at {n}^2 binary (unforced), FFTW replaced by the oracle FFT on "
              f"{thr} threads, reference loops single-threaded")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 5), "unit": "steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 / v, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"binary CHNS {n}^2 (reference etd2rk, CPU)", "grid": n},
        "cpu_baseline": {"value": round(v, 5), "unit": "steps/s", "kind": "reference", "cores": thr, "sample": sample},
        "e2e": {"value": round(v, 5), "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="chns", choices=["chns", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--dt", type=float, default=DT_DEFAULT)
    ap.add_argument("--accuracy-steps", type=int, default=1000)
    ap.add_argument("--precision", default="fp32_state64", choices=["fp32_state64", "fp32"],
                    help="headline mode: FP32 right-hand side with a float-pair state (default) or plain FP32")
    ap.add_argument("--other-steps", type=int, default=200,
                    help="steps of the throughput leg of the other FP32 mode (0: skip)")
    ap.add_argument("--no-adjoint", dest="adjoint", action="store_false")
    ap.add_argument("--ensemble-steps", type=int, default=500, help="steps of the ensemble leg (0: skip)")
    ap.add_argument("--no-ternary", dest="ternary", action="store_false",
                    help="skip the ternary leg (the ternary model at the bench grid, three precisions)")
    ap.add_argument("--adjoint-big-steps", type=int, default=1000,
                    help="steps of the 4096^2 FP32 adjoint memory check (0: skip)")
    ap.add_argument("--profile-case", nargs="?", const="step", default=None,
                    choices=["step", "step_state64", "adjoint", "adjoint_2048", "ensemble"],
                    help="only run a small fixed case for ncu captures (step: --steps steps of the FP32 "
                         "workload; step_state64: the same with CHNS_FP32_STATE64; adjoint; ensemble); "
                         "prints nothing")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.profile_case:
        run_profile_case(args)
        return
    if args.impl == "reference":
        if args.n == N_DEFAULT and args.steps > 10:
            args.steps = 10  # one reference step at 4096^2 takes seconds
            args.warmup = 3
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
