"""CPU tests of the C ABI library: it loads without a GPU, exports every
function include/chns.h declares, and validates arguments before touching CUDA."""
import ctypes
import math
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "chns.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(chns_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    import chns_b200

    if not os.path.isfile(chns_b200.LIB_PATH):
        pytest.fail("libchns_b200.so is not built (run __graft_entry__.build())")
    return chns_b200.load_library()


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert "chns_create" in names and "chns_step" in names and "chns_dfft_noalloc" in names
    for nm in names:
        assert hasattr(lib, nm), nm


def test_default_params_are_the_reference_defaults(lib):
    import chns_b200

    p = chns_b200.default_params(chns_b200.MODEL_BINARY, 1024)
    # global.h:20-31, 102-104
    assert p["lx"] == 4.0 * math.pi and p["dt"] == 1e-4 and p["nu"] == 0.01
    assert p["sigma"] == 2.0 and p["lambda"] == 1e-6 and p["epsilon"] == 3.0 * (4.0 * math.pi / 1024)
    q = chns_b200.default_params(chns_b200.MODEL_TERNARY, 1024)
    assert (q["sigma12"], q["sigma23"], q["sigma13"], q["lambda"], q["xlambda"]) == (0.2, 0.45, 0.2, 1e-4, 2.0)


@pytest.mark.parametrize("bad", [dict(nx=100), dict(nx=8192), dict(ny=512), dict(dealias_div=2.0),
                                 dict(dt=0.0), dict(model=3), dict(precision=7), dict(coef_mode=4),
                                 dict(force_amp=1.0, force_k=4.5)])
def test_create_rejects_bad_parameters_without_cuda(lib, bad):
    import chns_b200

    p = dict(model=1, nx=256, ny=256, dt=1e-3, nu=0.01, sigma=0.2, epsilon=0.05)
    p["lambda"] = 0.005
    p.update(bad)
    if "nx" in bad and "ny" not in bad:
        p["ny"] = bad["nx"]
    s = chns_b200.make_params(p)
    h = ctypes.c_void_p()
    rc = lib.chns_create(ctypes.byref(s), ctypes.byref(h))
    assert rc in (-1, -5) and not h.value


def test_noalloc_rejects_sizes_before_touching_the_device(lib):
    for n in (1024, 2048, 100, 16):
        assert lib.chns_dfft_noalloc(ctypes.c_void_p(8), ctypes.c_void_p(8), n, None) == -5
    assert lib.chns_dfft_noalloc(None, None, 64, None) == -1


def test_status_strings(lib):
    for s in (0, -1, -2, -3, -4, -5, -6, -7):
        assert lib.chns_status_string(s)
    assert lib.chns_status_string(-7) != lib.chns_status_string(-99)


def test_calls_reject_a_null_context_without_cuda(lib):
    for fn in ("chns_step", "chns_check", "chns_synchronize", "chns_launches_per_step", "chns_tma_tiles"):
        f = getattr(lib, fn)
        rc = f(None, 1) if fn == "chns_step" else f(None)
        assert rc in (-1, 0) if fn in ("chns_launches_per_step", "chns_tma_tiles") else rc == -1, fn


def test_binding_rejects_wrongly_shaped_host_arrays(lib):
    """The binding checks host array shapes before the C call reads nx * ny values
    from them (no GPU needed: the checks come first)."""
    import numpy as np

    import chns_b200

    c = chns_b200.Context.__new__(chns_b200.Context)
    c.L, c._h, c.model, c.nx, c.ny = lib, None, 1, 32, 32
    c.shape = (32, 17)
    with pytest.raises(ValueError):
        c.set_phase_real(np.zeros((32, 30)))
    with pytest.raises(ValueError):
        c.set_phase_real(np.zeros((32, 32)), np.zeros(32 * 32))
    with pytest.raises(ValueError):
        c.dfft(np.zeros((16, 32)))
    with pytest.raises(ValueError):
        c.set_state(np.zeros((32, 16), np.complex128))
    with pytest.raises(ValueError):
        c.adjoint(2, 1, loss_w=(1.0, 1.0))


@pytest.mark.parametrize("std,lang", [("c89", "c"), ("c99", "c"), ("c++11", "c++")])
def test_header_compiles_and_links_for_c_and_cpp_hosts(lib, tmp_path, std, lang):
    """include/chns.h is a plain C header: it compiles warning-free as C89, C99
    (pedantic) and C++11, and a host program links against the library and calls
    an entry point that needs no GPU."""
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "host.c"
    src.write_text('#include "chns.h"\n'
                   "int main(void) { chns_params p; chns_default_params(&p, CHNS_MODEL_BINARY, 256);\n"
                   "  return p.nx == 256 && p.ny == 256 ? 0 : 1; }\n")
    cc = "g++" if lang == "c++" else "gcc"
    libdir = os.path.join(root, "ternary-chns_b200", "lib")
    exe = tmp_path / "host"
    subprocess.run([cc, f"-std={std}", "-Wall", "-Wextra", "-Werror"] + (["-pedantic"] if std == "c99" else [])
                   + ["-x", lang, str(src), "-x", "none", "-I", os.path.join(root, "include"), "-L", libdir,
                      "-lchns_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True, capture_output=True)
    assert subprocess.run([str(exe)]).returncode == 0


def test_slab_plan_rejects_bad_decompositions_without_cuda(lib):
    """chns_slab_create validates the decomposition before it allocates."""
    from chns_b200 import slab

    slab._bind(lib)
    h = ctypes.c_void_p()
    assert lib.chns_slab_create(64, 3, 0, ctypes.byref(h)) == -1     # 64 x-rows do not split over 3 ranks
    assert lib.chns_slab_create(64, 64, 0, ctypes.byref(h)) == -1    # one x-row per rank: the y passes need pairs
    assert lib.chns_slab_create(64, 2, 2, ctypes.byref(h)) == -1     # rank out of range
    assert lib.chns_slab_create(8192, 2, 0, ctypes.byref(h)) == -5   # beyond the largest grid
    assert lib.chns_slab_create(96, 2, 0, ctypes.byref(h)) == -5     # not a power of two
    assert not h.value
