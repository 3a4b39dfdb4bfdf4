"""spectrum.c and perimeter.c on the device (chns_spectrum, chns_perimeter) against
the reference's own functions (oracle/_ref).  Spectra: FP64 relative <= 1e-12
per bin (positive sums in a different order), FP32 <= 1e-4 (or 1e-6 of the
largest bin); chns_spectrum leaves
the state as it was (spectrum.c truncates it in place).  Perimeter: the counts
recovered from the reference's %g output are equal, Sp_0 / Sp_t / def agree to
the 6 printed digits."""
import math
import tempfile

import numpy as np
import pytest

from _golden import load_small

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def chns():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import chns_b200

    chns_b200.load_library()
    return chns_b200


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("name", ["ns32", "bin32", "ter32", "bindef64", "terdef64", "nssf32", "binsf64", "tersf64"])
def test_spectrum_matches_reference(chns, name, prec):
    import oracle as O

    g = load_small(name)
    R = O.RefLib(name)
    R.set_state(*g["final"])
    want = R.spectrum(tempfile.mkdtemp())
    with chns.Context(dict(g["params"], precision=prec)) as c:
        c.set_state(*g["final"])
        before = c.get_state()
        got = c.spectrum()
        after = c.get_state()
    for a, b in zip(before, after):
        assert np.array_equal(a, b)
    assert set(got) == set(want)
    # FP32: bins far below the largest one carry FP32 rounding of the larger modes
    rtol, atol = (1e-12, 1e-14) if prec == 0 else (1e-4, 1e-6)
    for k in want:
        assert got[k].shape == want[k].shape, k
        scale = max(np.abs(want[k]).max(), 1e-300)
        assert np.allclose(got[k], want[k], rtol=rtol, atol=atol * scale), (k, np.abs(got[k] - want[k]).max())


def _drops(n, lx, centres, radius, eps):
    x = np.arange(n) * lx / n
    X, Y = np.meshgrid(x, x, indexing="ij")
    c = np.zeros((n, n))
    for cx, cy in centres:
        r = np.sqrt((X - cx) ** 2 + (Y - cy) ** 2)
        c += 0.5 * (1 - np.tanh((r - radius) / eps))
    return 0.02 + 0.9 * c


@pytest.mark.parametrize("name", ["bin32", "bindef64", "ter32", "terdef64"])
def test_perimeter_matches_reference(chns, name):
    import oracle as O

    g = load_small(name)
    p = g["params"]
    n, lx = p["nx"], p["lx"]
    eps = 2 * lx / n
    c1 = _drops(n, lx, [(0.3 * lx, 0.4 * lx), (0.75 * lx, 0.7 * lx)], 0.15 * lx, eps)
    ph = [c1] if p["model"] == 1 else [c1, _drops(n, lx, [(0.5 * lx, 0.2 * lx)], 0.2 * lx, eps)]
    R = O.RefLib(name)
    R.set_phase_real(*ph)
    want = R.perimeter()
    with chns.Context(p) as c:
        c.set_phase_real(*ph)
        got = c.perimeter()
    assert len(got) == len(want) == p["model"]
    dx = lx / n
    for gv, (t, sp0, spt, dfm) in zip(got, want):
        assert gv["count1"] == round(spt / dx)
        assert gv["count2"] == round((sp0 / 2) ** 2 / (math.pi * dx * dx))
        assert gv["count1"] > 0 and gv["count2"] > 0
        for a, b in ((gv["sp_0"], sp0), (gv["sp_t"], spt), (gv["def"], dfm)):
            assert abs(a - b) <= 1e-5 * abs(b) + 1e-12
