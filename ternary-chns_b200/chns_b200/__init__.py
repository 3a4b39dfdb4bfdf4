"""Host-side mirror of the reference's step interface over the C ABI (include/chns.h).

The reference advances the state with etd2rk(cwz, cphi[, cphi2]) in FFTW's
spectral layout (etd2rk.c:14-20); ``Context.step`` is that call on the GPU, with
the parameters of global.h passed explicitly (``params``) instead of compiled in.

Arrays are numpy: spectral fields (nx, ny//2+1) complex128 in FFTW layout,
real fields (nx, ny) float64.  There is no CPU fallback: without the built
library (ternary-chns_b200/lib/libchns_b200.so) or without a GPU every call
raises.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
# CHNS_B200_LIB names a variant build of the same library (e.g. one compiled
# with other CHNS_* defines by build.build(defines=..., lib=...)) for parity
# tests and timing of that variant; the default is the in-tree build.
LIB_PATH = os.environ.get("CHNS_B200_LIB") or os.path.join(PKG, "lib", "libchns_b200.so")

MODEL_NS, MODEL_BINARY, MODEL_TERNARY = 0, 1, 2
FP64, FP32, FP32_STATE64 = 0, 1, 2
COEF_REFERENCE, COEF_ACCURATE = 0, 1
# truncation: the sharp cut, or the reference's SMOOTH_FILTER build (functions.c:69-72)
FILTER_SHARP, FILTER_SMOOTH = 0, 1
HOST, DEVICE = 0, 1
INIT_W_ZERO, INIT_W_TAYLOR_GREEN, INIT_W_SHELL = 0, 1, 2
INIT_C_DROP, INIT_C_NOISE = 0, 1

STATUS = {0: "ok", -1: "bad argument", -2: "CUDA error", -3: "non-finite or blown-up state",
          -4: "device wait timed out", -5: "unsupported size or option", -6: "out of memory",
          -7: "file could not be read or written"}


class ChnsError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what}: {STATUS.get(status, status)} ({status})")
        self.status = status


class Params(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int), ("precision", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("dt", ctypes.c_double), ("nu", ctypes.c_double),
        ("lam", ctypes.c_double), ("sigma", ctypes.c_double), ("epsilon", ctypes.c_double),
        ("sigma12", ctypes.c_double), ("sigma13", ctypes.c_double), ("sigma23", ctypes.c_double),
        ("xlambda", ctypes.c_double), ("dealias_div", ctypes.c_double), ("coef_mode", ctypes.c_int),
        ("force_amp", ctypes.c_double), ("force_k", ctypes.c_double), ("filter", ctypes.c_int),
    ]


_lib = None


def load_library(path: str = LIB_PATH):
    """Loads libchns_b200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.isfile(path):
        raise FileNotFoundError(f"{path} is missing: run __graft_entry__.build() (no CPU fallback exists)")
    L = ctypes.CDLL(path)
    vp, dp, ip = ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int
    L.chns_default_params.argtypes = [ctypes.POINTER(Params), ip, ip]
    L.chns_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(vp)]
    L.chns_destroy.argtypes = [vp]
    L.chns_set_stream.argtypes = [vp, vp]
    L.chns_synchronize.argtypes = [vp]
    L.chns_set_state.argtypes = [vp, dp, dp, dp, ip]
    L.chns_get_state.argtypes = [vp, dp, dp, dp, ip]
    L.chns_set_phase_real.argtypes = [vp, dp, dp, ip]
    L.chns_step.argtypes = [vp, ip]
    L.chns_rhs.argtypes = [vp, dp, dp, dp, ip]
    L.chns_dfft.argtypes = [vp, dp, dp, ip]
    L.chns_ifft.argtypes = [vp, dp, dp, ip]
    L.chns_diagnostics.argtypes = [vp, dp, dp]
    L.chns_launches_per_step.argtypes = [vp]
    L.chns_tma_tiles.argtypes = [vp]
    L.chns_etd_coefficients.argtypes = [vp, ip, ip, vp]
    L.chns_truncation_rows.argtypes = [vp, vp]
    L.chns_profile_step.argtypes = [vp, ip, vp, vp, ip]
    L.chns_profile_step.restype = ip
    L.chns_adjoint.argtypes = [vp, ip, ip, vp, vp, vp, vp, vp, ip]
    L.chns_adjoint.restype = ip
    L.chns_pin_host.argtypes = [vp, vp, ctypes.c_size_t]
    L.chns_pin_host.restype = ip
    L.chns_unpin_host.argtypes = [vp, vp]
    L.chns_unpin_host.restype = ip
    L.chns_check.argtypes = [vp]
    L.chns_check.restype = ip
    L.chns_spectrum_shells.argtypes = [vp]
    L.chns_spectrum.argtypes = [vp, vp]
    L.chns_spectrum.restype = ip
    L.chns_perimeter.argtypes = [vp, vp]
    L.chns_perimeter.restype = ip
    L.chns_save.argtypes = [vp, ctypes.c_char_p]
    L.chns_save.restype = ip
    L.chns_load.argtypes = [vp, ctypes.c_char_p]
    L.chns_load.restype = ip
    L.chns_write_fields.argtypes = [vp, ctypes.c_char_p, ip, ip]
    L.chns_write_fields.restype = ip
    L.chns_read_phase.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p]
    L.chns_read_phase.restype = ip
    L.chns_init_vorticity.argtypes = [vp, ip, ctypes.c_double]
    L.chns_init_vorticity.restype = ip
    L.chns_init_phase.argtypes = [vp, ip, ctypes.c_uint]
    L.chns_init_phase.restype = ip
    L.chns_ensemble_create.argtypes = [vp, ip, ctypes.POINTER(vp)]
    L.chns_ensemble_create.restype = ip
    L.chns_ensemble_destroy.argtypes = [vp]
    L.chns_ensemble_member.argtypes = [vp, ip]
    L.chns_ensemble_member.restype = vp
    L.chns_ensemble_size.argtypes = [vp]
    L.chns_ensemble_step.argtypes = [vp, ip]
    L.chns_ensemble_step.restype = ip
    L.chns_ensemble_synchronize.argtypes = [vp]
    L.chns_ensemble_synchronize.restype = ip
    L.chns_ensemble_persistent.argtypes = [vp, ip]
    L.chns_ensemble_persistent.restype = ip
    L.chns_dfft_noalloc.argtypes = [vp, vp, ip, vp]
    L.chns_dfft_noalloc.restype = ip
    L.chns_tune_override.argtypes = [ip, ip]
    L.chns_tune_override.restype = ip
    L.chns_truncation_factor.argtypes = [vp, ip, ip, vp]
    L.chns_truncation_factor.restype = ip
    L.chns_status_string.restype = ctypes.c_char_p
    L.chns_status_string.argtypes = [ip]
    _lib = L
    return L


# chns_tune_override knobs: rows per TMA box of the row kernels' tiles; P1 with two CTAs per
# row; grad c kept in real space from P2 for P4; stage kernels as programmatic dependent launches
TUNE_TMA_BOX_ROWS, TUNE_P1_SPLIT, TUNE_P4_GRAD, TUNE_PDL = 1, 2, 3, 4


def tune_override(knob: int, value: int) -> None:
    """Overrides a launch-shape choice of the tuned tables for contexts created
    afterwards in this process (value -1: the table); results stay bitwise the same."""
    _check(load_library().chns_tune_override(int(knob), int(value)), "chns_tune_override")


def default_params(model: int, n: int) -> dict:
    """The reference's global.h defaults for `model` on an n x n grid."""
    L = load_library()
    s = Params()
    L.chns_default_params(ctypes.byref(s), model, n)
    return params_to_dict(s)


def params_to_dict(s: Params) -> dict:
    d = {k: getattr(s, k) for k, _ in Params._fields_}
    d["lambda"] = d.pop("lam")
    return d


def make_params(p: dict) -> Params:
    s = Params()
    s.model = int(p["model"])
    s.precision = int(p.get("precision", FP64))
    s.nx = int(p["nx"])
    s.ny = int(p.get("ny", p["nx"]))
    s.lx = float(p.get("lx", 2 * math.pi))
    s.ly = float(p.get("ly", s.lx))
    s.dt = float(p["dt"])
    s.nu = float(p.get("nu", 0.0))
    s.lam = float(p.get("lambda", 0.0))
    s.sigma = float(p.get("sigma", 0.0))
    s.epsilon = float(p.get("epsilon", 0.0))
    s.sigma12 = float(p.get("sigma12", 0.0))
    s.sigma13 = float(p.get("sigma13", 0.0))
    s.sigma23 = float(p.get("sigma23", 0.0))
    s.xlambda = float(p.get("xlambda", 2.0))
    s.dealias_div = float(p.get("dealias_div", 4.0))
    s.coef_mode = int(p.get("coef_mode", COEF_REFERENCE))
    s.force_amp = float(p.get("force_amp", 0.0))
    s.force_k = float(p.get("force_k", 0.0))
    s.filter = int(p.get("filter", FILTER_SHARP))
    return s


def _check(rc: int, what: str):
    if rc != 0:
        raise ChnsError(rc, what)


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class Context:
    """One simulation on one GPU: the reference's state (cwz, cphi / cphi1, cphi2)
    and its ETD2RK step."""

    def __init__(self, params: dict):
        self.L = load_library()
        self.params = dict(params)
        self._p = make_params(params)
        h = ctypes.c_void_p()
        _check(self.L.chns_create(ctypes.byref(self._p), ctypes.byref(h)), "chns_create")
        self._h = h
        self.model = self._p.model
        self.nx, self.ny = self._p.nx, self._p.ny
        self.shape = (self.nx, self.ny // 2 + 1)

    def close(self):
        if getattr(self, "_h", None):
            self.L.chns_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def _spec(self, a):
        a = np.ascontiguousarray(a, np.complex128)
        if a.shape != self.shape:
            raise ValueError(f"expected spectral shape {self.shape}, got {a.shape}")
        return a

    def _real(self, a):
        a = np.ascontiguousarray(a, np.float64)
        if a.shape != (self.nx, self.ny):
            raise ValueError(f"expected real shape {(self.nx, self.ny)}, got {a.shape}")
        return a

    def set_state(self, w, c1=None, c2=None):
        arrs = [self._spec(a) if a is not None else None for a in (w, c1, c2)]
        _check(self.L.chns_set_state(self._h, *[_ptr(a) for a in arrs], HOST), "chns_set_state")

    def get_state(self):
        out = [np.empty(self.shape, np.complex128) for _ in range(self.model + 1)]
        ptrs = [_ptr(a) for a in out] + [None] * (3 - len(out))
        _check(self.L.chns_get_state(self._h, *ptrs, HOST), "chns_get_state")
        return out

    def set_phase_real(self, p1, p2=None):
        a = self._real(p1)
        b = self._real(p2) if p2 is not None else None
        _check(self.L.chns_set_phase_real(self._h, _ptr(a), _ptr(b), HOST), "chns_set_phase_real")

    def pin_host(self, a: np.ndarray):
        """Page-locks a numpy array passed to set_state / get_state on every step
        (until unpin_host or close; the array must stay alive until then)."""
        _check(self.L.chns_pin_host(self._h, ctypes.c_void_p(a.ctypes.data), a.nbytes), "chns_pin_host")

    def unpin_host(self, a: np.ndarray):
        _check(self.L.chns_unpin_host(self._h, ctypes.c_void_p(a.ctypes.data)), "chns_unpin_host")

    def check(self):
        """Raises ChnsError (status -3) if the state holds NaN or infinite values."""
        _check(self.L.chns_check(self._h), "chns_check")

    def spectrum(self) -> dict:
        """spectrum.c's shell spectra (ek, ensk, sph | sph1, sph2, sp12, ekx, eky);
        the state is not modified."""
        ns = self.L.chns_spectrum_shells(self._h)
        nph = {0: 0, 1: 1, 2: 3}[self.model]
        out = np.zeros((2 + nph) * ns + 2 * (self.nx // 2 + 1))
        _check(self.L.chns_spectrum(self._h, _ptr(out)), "chns_spectrum")
        o = {"ek": out[:ns], "ensk": out[ns:2 * ns]}
        for k, nm in enumerate({1: ["sph"], 2: ["sph1", "sph2", "sp12"]}.get(self.model, [])):
            o[nm] = out[(2 + k) * ns:(3 + k) * ns]
        b = (2 + nph) * ns
        o["ekx"] = out[b:b + self.nx // 2 + 1]
        o["eky"] = out[b + self.nx // 2 + 1:]
        return o

    def perimeter(self) -> list:
        """perimeter.c per phase field: dict(count1, count2, sp_0, sp_t, def)."""
        out = np.zeros(10)
        _check(self.L.chns_perimeter(self._h, _ptr(out)), "chns_perimeter")
        keys = ("count1", "count2", "sp_0", "sp_t", "def")
        return [dict(zip(keys, out[5 * f:5 * f + 5])) for f in range(self.model)]

    def save(self, path: str):
        """Checkpoint: parameters and spectral state, for a bit-exact resume."""
        _check(self.L.chns_save(self._h, os.fsencode(path)), "chns_save")

    def load(self, path: str):
        """Resume from a chns_save file written with the same parameters."""
        _check(self.L.chns_load(self._h, os.fsencode(path)), "chns_load")

    def write_fields(self, directory: str, index: int, truncate: bool = False):
        """main.c's dumps: <directory>/vort/wz.<index>, phase_field/phi[1|2].<index>,
        raw FP64 nx x ny (write_array.c); truncate=True as DUMP_REAL_MPI."""
        _check(self.L.chns_write_fields(self._h, os.fsencode(directory), int(index), int(bool(truncate))),
               "chns_write_fields")

    def read_phase(self, path1: str, path2: str | None = None):
        """INIT_READ_DATA: raw FP64 nx x ny phase file(s) (read_array.c), dfft, truncation."""
        _check(self.L.chns_read_phase(self._h, os.fsencode(path1), os.fsencode(path2) if path2 else None),
               "chns_read_phase")

    def init_vorticity(self, kind: int = INIT_W_ZERO, amplitude: float = 1.0):
        """init.c's vorticity on the device: zero or Taylor-Green (TG_INIT)."""
        _check(self.L.chns_init_vorticity(self._h, int(kind), float(amplitude)), "chns_init_vorticity")

    def init_phase(self, kind: int, seed: int = 10):
        """init.c's phase fields on the device: the binary drop or the ternary noise
        (the C library's rand() after srand(seed); the reference seeds 10 + 2 rank)."""
        _check(self.L.chns_init_phase(self._h, int(kind), int(seed)), "chns_init_phase")

    def step(self, n: int = 1):
        _check(self.L.chns_step(self._h, int(n)), "chns_step")

    def synchronize(self):
        _check(self.L.chns_synchronize(self._h), "chns_synchronize")

    def rhs(self):
        out = [np.empty(self.shape, np.complex128) for _ in range(self.model + 1)]
        ptrs = [_ptr(a) for a in out] + [None] * (3 - len(out))
        _check(self.L.chns_rhs(self._h, *ptrs, HOST), "chns_rhs")
        return out

    def dfft(self, real):
        x = self._real(real)
        out = np.empty(self.shape, np.complex128)
        _check(self.L.chns_dfft(self._h, _ptr(x), _ptr(out), HOST), "chns_dfft")
        return out

    def ifft(self, spec):
        s = self._spec(spec)
        out = np.empty((self.nx, self.ny), np.float64)
        _check(self.L.chns_ifft(self._h, _ptr(s), _ptr(out), HOST), "chns_ifft")
        return out

    def diagnostics(self):
        """((bulk, gradient) free energy, (<|u|^2/2>, phase-1 mean, phase-2 mean)) of the state."""
        fe = np.zeros(2)
        ke = np.zeros(3)
        rc = self.L.chns_diagnostics(self._h, _ptr(fe), _ptr(ke))
        if rc not in (0, -3):
            _check(rc, "chns_diagnostics")
        return fe, ke, rc

    def adjoint(self, nsteps: int, ckpt: int = 20, loss_w=(1.0, 1.0, 1.0)):
        """Discrete adjoint of `nsteps` ETD2RK steps from the current state.  Returns
        (J, dJ/d omega_hat_0, dJ/d c_hat_0, dJ/d params): for the binary model
        dJ/d c_hat_0 is one array and the parameters are (nu, lambda, sigma); for the
        ternary model it is a pair (c1, c2) and the parameters are (nu, lambda,
        sigma_12, sigma_13, sigma_23); for pure Navier-Stokes (loss_w[0] kinetic
        energy, loss_w[1] enstrophy) it is None and the parameters are (nu, 0, 0).
        The state is unchanged."""
        lw = np.ascontiguousarray(loss_w, np.float64)
        if lw.shape != (3,):
            raise ValueError("loss_w: three weights")
        J = np.zeros(1)
        gw = np.empty(self.shape, np.complex128)
        nc = max(self.model, 1)
        gc = np.empty((nc,) + self.shape, np.complex128)
        gp = np.zeros(5 if self.model == MODEL_TERNARY else 3)
        _check(self.L.chns_adjoint(self._h, int(nsteps), int(ckpt), _ptr(lw), _ptr(J), _ptr(gw), _ptr(gc),
                                   _ptr(gp), HOST), "chns_adjoint")
        if self.model == MODEL_NS:
            return float(J[0]), gw, None, gp
        return float(J[0]), gw, (gc[0] if self.model == MODEL_BINARY else (gc[0], gc[1])), gp

    def launches_per_step(self) -> int:
        return self.L.chns_launches_per_step(self._h)

    def tma_tiles(self) -> bool:
        """True when the step's row kernels load their tiles with TMA."""
        return bool(self.L.chns_tma_tiles(self._h))


class Member(Context):
    """A member of an Ensemble: the Context calls on a context the ensemble owns."""

    def __init__(self, ens: "Ensemble", index: int, params: dict):
        self.L = ens.L
        self.params = dict(params)
        self._p = make_params(params)
        h = self.L.chns_ensemble_member(ens._h, index)
        if not h:
            raise ChnsError(-1, "chns_ensemble_member")
        self._h = ctypes.c_void_p(h)
        self.model = self._p.model
        self.nx, self.ny = self._p.nx, self._p.ny
        self.shape = (self.nx, self.ny // 2 + 1)

    def close(self):
        self._h = None  # owned by the ensemble


class Ensemble:
    """Independent runs (any mix of models, sizes, precisions and parameters)
    advanced together by chns_ensemble_step: one CUDA graph launch per step with
    every member on its own branch, or (``persistent = True``, when every member
    is a ternary FP32 run at 256^2..1024^2) one persistent kernel per step.
    ``members[i]`` behaves like a Context."""

    def __init__(self, params_list):
        self.L = load_library()
        plist = list(params_list)
        arr = (Params * len(plist))(*[make_params(p) for p in plist])
        h = ctypes.c_void_p()
        _check(self.L.chns_ensemble_create(ctypes.cast(arr, ctypes.c_void_p), len(plist), ctypes.byref(h)),
               "chns_ensemble_create")
        self._h = h
        self.members = [Member(self, i, p) for i, p in enumerate(plist)]

    def __len__(self):
        return len(self.members)

    def step(self, n: int = 1):
        _check(self.L.chns_ensemble_step(self._h, int(n)), "chns_ensemble_step")

    def synchronize(self):
        _check(self.L.chns_ensemble_synchronize(self._h), "chns_ensemble_synchronize")

    @property
    def persistent(self) -> bool:
        """True when a step is one persistent kernel over all members."""
        rc = self.L.chns_ensemble_persistent(self._h, -1)
        _check(min(rc, 0), "chns_ensemble_persistent")
        return rc == 1

    @persistent.setter
    def persistent(self, enable: bool):
        rc = self.L.chns_ensemble_persistent(self._h, 1 if enable else 0)
        _check(min(rc, 0), "chns_ensemble_persistent")

    def close(self):
        if getattr(self, "_h", None):
            for m in self.members:
                m._h = None
            self.L.chns_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
