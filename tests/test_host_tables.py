"""The host-side tables of chns_create (ETD coefficients, truncation rows, the
SMOOTH_FILTER factors), read through chns_etd_coefficients / chns_truncation_rows /
chns_truncation_factor without a GPU, against the C restatement of the reference
(orc_etd_coefs: etd2rk.c:88-206; orc_truncation: functions.c:47-84) on every mode
of the small golden configurations, in both coefficient modes.  Bitwise: both
compute in double with the reference's operand order and without contraction."""
import ctypes

import numpy as np
import pytest

import oracle as O
from _golden import load_small


@pytest.fixture(scope="module")
def chns():
    import chns_b200

    L = chns_b200.load_library()
    L.chns_etd_coefficients.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    L.chns_truncation_rows.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.chns_truncation_factor.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    O.build_oracle_lib()
    return chns_b200, L


CASES = [(name, mode) for name in ("ns32", "bin64", "ter64", "bindef64", "terdef64") for mode in (0, 1)]


@pytest.mark.parametrize("name,mode", CASES)
def test_etd_coefficients_equal_the_restatement(chns, name, mode):
    C, L = chns
    p = dict(load_small(name)["params"], coef_mode=mode)
    prm = C.make_params(p)
    o = O.Oracle(p)
    n = p["nx"]
    out = np.zeros(6)
    for i in range(n):
        for j in range(n // 2 + 1):
            assert L.chns_etd_coefficients(ctypes.byref(prm), i, j, out.ctypes.data) == 0
            assert np.array_equal(out, np.array(o.etd_coefs(i, j))), (name, mode, i, j)


@pytest.mark.parametrize("name", ["ns32", "bin64", "ter64", "bindef64"])
def test_truncation_rows_equal_the_restatement(chns, name):
    C, L = chns
    p = load_small(name)["params"]
    n = p["nx"]
    mrow = np.full(n // 2 + 1, -7, np.int32)
    assert L.chns_truncation_rows(ctypes.byref(C.make_params(p)), mrow.ctypes.data) == 0
    kept = O.Oracle(p).truncation(np.ones((n, n // 2 + 1), np.complex128)) != 0
    for j in range(n // 2 + 1):
        ms = [m for m in range(n // 2 + 1) if kept[m, j]]
        want = max(ms) if ms else -1
        assert mrow[j] == want, (name, j)
        # the cut is symmetric in kx: |m| <= mrow[j] on both sides
        assert all(kept[(-m) % n, j] for m in range(want + 1))


@pytest.mark.parametrize("name", ["nssf32", "binsf64", "tersf64", "binsfdef64"])
def test_smooth_filter_keeps_every_row(chns, name):
    C, L = chns
    p = load_small(name)["params"]
    assert p["filter"] == C.FILTER_SMOOTH
    n = p["nx"]
    mrow = np.full(n // 2 + 1, -7, np.int32)
    assert L.chns_truncation_rows(ctypes.byref(C.make_params(p)), mrow.ctypes.data) == 0
    assert np.all(mrow == n // 2)


@pytest.mark.parametrize("name", ["bin64", "bindef64", "nssf32", "binsf64", "tersf64", "binsfdef64"])
def test_truncation_factors_equal_the_restatement(chns, name):
    """One truncation() of a field of ones is f * f per mode (SMOOTH_FILTER's two
    products, functions.c:69-72) or the 0/1 mask of the sharp cut (:74-79)."""
    C, L = chns
    p = load_small(name)["params"]
    prm = C.make_params(p)
    n = p["nx"]
    tr = O.Oracle(p).truncation(np.ones((n, n // 2 + 1), np.complex128))
    assert not np.any(tr.imag)
    f = np.zeros(1)
    got = np.zeros((n, n // 2 + 1))
    for i in range(n):
        for j in range(n // 2 + 1):
            assert L.chns_truncation_factor(ctypes.byref(prm), i, j, f.ctypes.data) == 0
            got[i, j] = (1.0 * f[0]) * f[0]
    assert np.array_equal(got, tr.real), name
    if p.get("filter"):
        assert got[0, 0] == 1.0 and 0.0 < got.min() < 1e-30  # the corner (n/2, n/2): exp(-36)^2


def test_tune_override_checks_its_arguments(chns):
    C, L = chns
    for knob, bad in ((C.TUNE_TMA_BOX_ROWS, (0, 4, 12, 264, -2)), (C.TUNE_P1_SPLIT, (2, -2)),
                      (C.TUNE_P4_GRAD, (2, -2)), (C.TUNE_PDL, (2, -2)), (7, (1,))):
        for v in bad:
            assert L.chns_tune_override(knob, v) == -1, (knob, v)
    for knob, good in ((C.TUNE_TMA_BOX_ROWS, (8, 64, 256, -1)), (C.TUNE_P1_SPLIT, (0, 1, -1)),
                       (C.TUNE_P4_GRAD, (0, 1, -1)), (C.TUNE_PDL, (0, 1, -1))):
        for v in good:
            assert L.chns_tune_override(knob, v) == 0, (knob, v)


def test_tables_reject_bad_arguments(chns):
    C, L = chns
    p = C.make_params(load_small("bin64")["params"])
    out = np.zeros(6)
    assert L.chns_etd_coefficients(ctypes.byref(p), 64, 0, out.ctypes.data) == -1
    assert L.chns_etd_coefficients(ctypes.byref(p), 0, 33, out.ctypes.data) == -1
    assert L.chns_etd_coefficients(ctypes.byref(p), 0, 0, None) == -1
    assert L.chns_truncation_rows(ctypes.byref(p), None) == -1
    assert L.chns_truncation_factor(ctypes.byref(p), 0, 33, out.ctypes.data) == -1
    assert L.chns_truncation_factor(ctypes.byref(p), 0, 0, None) == -1
    q = C.make_params(dict(load_small("bin64")["params"], filter=2))
    assert L.chns_truncation_factor(ctypes.byref(q), 0, 0, out.ctypes.data) == -1
    bad = C.make_params(dict(load_small("bin64")["params"], nx=100, ny=100))
    assert L.chns_truncation_rows(ctypes.byref(bad), out.ctypes.data) != 0
