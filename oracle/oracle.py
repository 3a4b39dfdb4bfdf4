"""ctypes front-end to the oracle (test infrastructure only).

Two checkers live under oracle/:

* ``Oracle``  -- the C restatement of the reference's step (chns_oracle.c) with
  run-time parameters, built into oracle/liboracle.so.
* ``RefLib``  -- the reference's own sources compiled per configuration
  (oracle/build_ref.py -> oracle/_ref/<config>/libref.so), driven through
  oracle/ref_harness.c.

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline may import this
module.  Nothing in the product imports it.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

MODEL_NS, MODEL_BINARY, MODEL_TERNARY = 0, 1, 2


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double),
        ("dt", ctypes.c_double), ("nu", ctypes.c_double),
        ("lam", ctypes.c_double), ("sigma", ctypes.c_double), ("epsilon", ctypes.c_double),
        ("sigma12", ctypes.c_double), ("sigma13", ctypes.c_double), ("sigma23", ctypes.c_double),
        ("xlambda", ctypes.c_double), ("dealias_div", ctypes.c_double),
        ("coef_mode", ctypes.c_int), ("force_amp", ctypes.c_double), ("force_k", ctypes.c_double),
        ("filter", ctypes.c_int),
    ]


def build_oracle_lib(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("chns_oracle.c", "fft_cpu.c", "chns_oracle.h", "fft_cpu.h")]
    if not force and os.path.isfile(LIB) and all(os.path.getmtime(s) <= os.path.getmtime(LIB) for s in srcs):
        return LIB
    cc = os.environ.get("CC", "gcc")
    tmp = LIB + ".tmp"
    subprocess.check_call([cc, "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-std=gnu99",
                           "-o", tmp, srcs[0], srcs[1], "-lm", "-lpthread"])
    os.replace(tmp, LIB)
    return LIB


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.isfile(LIB):
            build_oracle_lib()
        L = ctypes.CDLL(LIB)
        vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int
        L.orc_create.restype = vp
        L.orc_create.argtypes = [ctypes.POINTER(OrcParams), ip]
        L.orc_destroy.argtypes = [vp]
        for f in ("orc_set_state", "orc_get_state", "orc_rhs"):
            getattr(L, f).argtypes = [vp, vp, vp, vp]
        L.orc_set_phase_real.argtypes = [vp, vp, vp]
        L.orc_step.argtypes = [vp, ip]
        L.orc_free_energy.argtypes = [vp, dp, dp]
        L.orc_kinetic_energy.argtypes = [vp, dp]
        L.orc_kinetic_energy.restype = ip
        for f in ("orc_dfft", "orc_ifft", "orc_truncation"):
            getattr(L, f).argtypes = [vp, vp]
        L.orc_etd_coefs.argtypes = [vp, ip, ip, dp]
        L.fftc_set_threads.argtypes = [ip]
        L.fftc_set_variant.argtypes = [ip]
        _lib = L
    return _lib


def set_fft_variant(v: int) -> None:
    """Selects the oracle FFT's rounding order (0: default radix-4, paired rows;
    1: radix-2, single rows) for every Oracle in this process."""
    _load().fftc_set_variant(int(v))


def _ptr(a):
    return None if a is None else a.ctypes.data


class Oracle:
    """C restatement of the reference step, with run-time parameters (dict as in params())."""

    def __init__(self, p: dict, nthreads: int = 1):
        self.p = dict(p)
        L = _load()
        self._L = L
        s = OrcParams(model=p["model"], nx=p["nx"], ny=p["ny"], lx=p["lx"], ly=p["ly"], dt=p["dt"],
                      nu=p["nu"], lam=p.get("lambda", 0.0), sigma=p.get("sigma", 0.0),
                      epsilon=p.get("epsilon", 0.0), sigma12=p.get("sigma12", 0.0),
                      sigma13=p.get("sigma13", 0.0), sigma23=p.get("sigma23", 0.0),
                      xlambda=p.get("xlambda", 2.0), dealias_div=p.get("dealias_div", 4.0),
                      coef_mode=p.get("coef_mode", 0), force_amp=p.get("force_amp", 0.0),
                      force_k=p.get("force_k", 0.0), filter=p.get("filter", 0))
        self._h = L.orc_create(ctypes.byref(s), nthreads)
        if not self._h:
            raise ValueError("oracle: bad parameters")
        self.nx, self.ny = p["nx"], p["ny"]
        self.shape = (self.nx, self.ny // 2 + 1)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.orc_destroy(h)
            self._h = None

    def _buf(self):
        return np.zeros(self.shape, np.complex128)

    def set_state(self, w, c1=None, c2=None):
        arrs = [np.ascontiguousarray(a, np.complex128) if a is not None else None for a in (w, c1, c2)]
        self._L.orc_set_state(self._h, *[_ptr(a) for a in arrs])

    def get_state(self):
        w, c1, c2 = self._buf(), self._buf(), self._buf()
        self._L.orc_get_state(self._h, _ptr(w), _ptr(c1), _ptr(c2))
        return [w, c1, c2][: 1 + self.p["model"]]

    def set_phase_real(self, p1, p2=None):
        a = np.ascontiguousarray(p1, np.float64)
        b = np.ascontiguousarray(p2, np.float64) if p2 is not None else None
        self._L.orc_set_phase_real(self._h, _ptr(a), _ptr(b))

    def step(self, n: int):
        self._L.orc_step(self._h, int(n))

    def rhs(self):
        w, c1, c2 = self._buf(), self._buf(), self._buf()
        self._L.orc_rhs(self._h, _ptr(w), _ptr(c1), _ptr(c2))
        return [w, c1, c2][: 1 + self.p["model"]]

    def free_energy(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        self._L.orc_free_energy(self._h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def kinetic_energy(self):
        out = (ctypes.c_double * 3)()
        n = self._L.orc_kinetic_energy(self._h, out)
        return list(out)[:n]

    def dfft(self, real):
        """real: (nx, ny) -> spectral (nx, ny/2+1), unnormalised (fft.c:11-14)."""
        buf = np.zeros((self.nx, self.ny + 2))
        buf[:, : self.ny] = real
        self._L.orc_dfft(self._h, buf.ctypes.data)
        return buf.view(np.complex128).copy()

    def ifft(self, spec):
        """spectral -> real, c2r then 1/(nx ny) (fft.c:16-31)."""
        buf = np.ascontiguousarray(spec, np.complex128).copy().view(np.float64).reshape(self.nx, self.ny + 2)
        buf = buf.copy()
        self._L.orc_ifft(self._h, buf.ctypes.data)
        return buf[:, : self.ny].copy()

    def truncation(self, spec):
        a = np.ascontiguousarray(spec, np.complex128).copy()
        self._L.orc_truncation(self._h, a.ctypes.data)
        return a

    def etd_coefs(self, i, j):
        out = (ctypes.c_double * 6)()
        self._L.orc_etd_coefs(self._h, i, j, out)
        return list(out)


# ---------------------------------------------------------------------------
# the reference compiled as a library
# ---------------------------------------------------------------------------

def _ref_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("chns_build_ref", os.path.join(HERE, "build_ref.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


build_ref = _ref_module()


def eval_ref_expr(expr: str, n: int, lx: float | None = None) -> float:
    """Evaluates one of build_ref.CONFIGS' C expressions with IEEE doubles, in C's order."""
    env = {"pi": math.pi}
    if lx is not None:
        env["dx"] = lx / n
        env["dy"] = lx / n
    return float(eval(expr, {"__builtins__": {}}, env))


def ref_config_params(name: str) -> dict:
    """The run-time parameter dict equal, bit for bit, to the compiled reference configuration."""
    cfg = build_ref.CONFIGS[name]
    n = cfg["n"]
    lx = eval_ref_expr(cfg["lx"], n)
    p = dict(model=cfg["model"], nx=n, ny=n, lx=lx, ly=lx,
             dt=eval_ref_expr(cfg["dt"], n), nu=eval_ref_expr(cfg["nu"], n))
    if cfg["model"] >= 1:
        p["epsilon"] = eval_ref_expr(cfg["eps"], n, lx)
        p["lambda"] = eval_ref_expr(cfg["lam"], n)
    if cfg["model"] == 1:
        p["sigma"] = eval_ref_expr(cfg["sigma"], n)
    if cfg["model"] == 2:
        p["sigma12"] = eval_ref_expr(cfg["s12"], n)
        p["sigma13"] = eval_ref_expr(cfg["s13"], n)
        p["sigma23"] = eval_ref_expr(cfg["s23"], n)
        p["xlambda"] = eval_ref_expr(cfg["xlam"], n)
    if cfg.get("filter"):
        p["filter"] = 1
    return p


class RefLib:
    """The reference's own etd2rk/nonlin/... compiled for one configuration (oracle/_ref)."""

    def __init__(self, name: str, nthreads: int = 1, dropin: bool = False):
        path = build_ref.lib_path(name, dropin)
        if not os.path.isfile(path):
            raise FileNotFoundError(path)
        L = ctypes.CDLL(path, mode=getattr(os, "RTLD_LOCAL", 0) | getattr(os, "RTLD_NOW", 2))
        vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int
        L.ref_setup.argtypes = [ip]
        L.ref_param.restype = ctypes.c_double
        L.ref_param.argtypes = [ctypes.c_char_p]
        for f in ("ref_set_state", "ref_get_state", "ref_rhs", "ref_get_velocity"):
            getattr(L, f).argtypes = [vp, vp, vp] if f != "ref_get_velocity" else [vp, vp, vp]
        L.ref_set_phase_real.argtypes = [vp, vp]
        L.ref_step.argtypes = [ip]
        L.ref_free_energy.argtypes = [dp, dp]
        L.ref_kinetic_energy.argtypes = [dp, ip]
        for f in ("ref_dfft", "ref_ifft", "ref_truncation"):
            getattr(L, f).argtypes = [vp]
        L.ref_set_time.argtypes = [ctypes.c_double]
        L.ref_setup(nthreads)
        self._L = L
        self.name = name
        self.model = L.ref_model()
        self.nx, self.ny = L.ref_nx(), L.ref_ny()
        self.shape = (self.nx, self.ny // 2 + 1)

    def param(self, key: str) -> float:
        return self._L.ref_param(key.encode())

    def _buf(self):
        return np.zeros(self.shape, np.complex128)

    def set_state(self, w, c1=None, c2=None):
        arrs = [np.ascontiguousarray(a, np.complex128) if a is not None else None for a in (w, c1, c2)]
        self._L.ref_set_state(*[_ptr(a) for a in arrs])

    def get_state(self):
        w, c1, c2 = self._buf(), self._buf(), self._buf()
        self._L.ref_get_state(_ptr(w), _ptr(c1), _ptr(c2))
        return [w, c1, c2][: 1 + self.model]

    def set_phase_real(self, p1, p2=None):
        a = np.ascontiguousarray(p1, np.float64)
        b = np.ascontiguousarray(p2, np.float64) if p2 is not None else None
        self._L.ref_set_phase_real(_ptr(a), _ptr(b))

    def step(self, n: int):
        self._L.ref_step(int(n))

    def rhs(self):
        w, c1, c2 = self._buf(), self._buf(), self._buf()
        self._L.ref_rhs(_ptr(w), _ptr(c1), _ptr(c2))
        return [w, c1, c2][: 1 + self.model]

    def free_energy(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        if self._L.ref_free_energy(ctypes.byref(a), ctypes.byref(b)) != 0:
            raise RuntimeError("free_energy output not parsed")
        return a.value, b.value

    def kinetic_energy(self):
        out = (ctypes.c_double * 4)()
        n = self._L.ref_kinetic_energy(out, 4)
        return list(out)[1:n]

    def spectrum(self, workdir: str) -> dict:
        """spectrum.c on the current state (state unchanged), run in `workdir`."""
        L = self._L
        L.ref_spectrum.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
        nshell = int(round(self.nx / math.sqrt(2.0) + 1.0))
        nph = {0: 0, 1: 1, 2: 3}[self.model]
        out = np.zeros((2 + nph) * nshell + (self.nx // 2 + 1) + (self.ny // 2 + 1))
        n = L.ref_spectrum(os.fsencode(workdir), out.ctypes.data)
        if n != nshell:
            raise RuntimeError("ref_spectrum failed")
        o = {"ek": out[:nshell], "ensk": out[nshell:2 * nshell]}
        names = {1: ["sph"], 2: ["sph1", "sph2", "sp12"]}.get(self.model, [])
        for k, nm in enumerate(names):
            o[nm] = out[(2 + k) * nshell:(3 + k) * nshell]
        b = (2 + nph) * nshell
        o["ekx"] = out[b:b + self.nx // 2 + 1]
        o["eky"] = out[b + self.nx // 2 + 1:]
        return o

    def last_line(self, which: int) -> str:
        """The last line the reference printed to a log (0 free_en_t.dat, 1 ken_t.dat,
        2 gamma.dat / gamma1.dat, 3 gamma2.dat)."""
        L = self._L
        L.ref_last_line.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        buf = ctypes.create_string_buffer(4096)
        n = L.ref_last_line(which, buf, 4096)
        if n < 0:
            raise RuntimeError("no line")
        return buf.value.decode()

    def perimeter(self) -> list:
        """perimeter.c on the current state: (t, Sp_0, Sp_t, def) per phase field,
        as printed with %g."""
        L = self._L
        L.ref_perimeter.argtypes = [ctypes.c_void_p]
        out = np.zeros(8)
        n = L.ref_perimeter(out.ctypes.data)
        return [list(out[k:k + 4]) for k in range(0, n, 4)]

    def dfft(self, real):
        buf = np.zeros((self.nx, self.ny + 2))
        buf[:, : self.ny] = real
        self._L.ref_dfft(buf.ctypes.data)
        return buf.view(np.complex128).copy()

    def ifft(self, spec):
        buf = np.ascontiguousarray(spec, np.complex128).copy().view(np.float64).reshape(self.nx, self.ny + 2).copy()
        self._L.ref_ifft(buf.ctypes.data)
        return buf[:, : self.ny].copy()

    def truncation(self, spec):
        a = np.ascontiguousarray(spec, np.complex128).copy()
        self._L.ref_truncation(a.ctypes.data)
        return a


def set_threads(n: int):
    _load().fftc_set_threads(int(n))
