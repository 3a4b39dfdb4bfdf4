"""The log files of chns_b200.logs have the reference's own text formats: lines
formatted from the values the reference printed equal the reference's lines, and
spectra formatted from the reference's spectrum arrays equal the files its
spectrum() wrote, byte for byte (the reference compiled here; no GPU)."""
import math
import os

import pytest

from _golden import load_small


def _values(line):
    return [float(x) for x in line.split()]


@pytest.mark.parametrize("name", ["ns32", "bin32", "ter32", "bindef64", "terdef64"])
def test_formats_equal_the_reference(name, tmp_path):
    import oracle as O
    from chns_b200 import logs

    g = load_small(name)
    p = g["params"]
    R = O.RefLib(name)
    R.set_state(*g["final"])
    R._L.ref_set_time(0.125)
    model = p["model"]
    if model >= 1:
        R.free_energy()
        line = R.last_line(0)
        v = _values(line)
        assert logs.free_energy_line(v[0], v[1:]) == line + "\n"
    R.kinetic_energy()
    line = R.last_line(1)
    v = _values(line)
    assert logs.kinetic_energy_line(v[0], model, v[1:]) == line + "\n"
    if model >= 1:
        R.perimeter()
        for k in range(model):
            line = R.last_line(2 + k)
            v = [float(x) if x != "-nan" else math.nan for x in line.split()]
            if any(math.isnan(x) for x in v):
                continue  # no phase above 0.5: %g prints -nan, Python nan
            assert logs.perimeter_line(v[0], dict(sp_0=v[1], sp_t=v[2], **{"def": v[3]})) == line + "\n"
    spec = R.spectrum(str(tmp_path))
    s, xs, ys = logs.spectrum_text(spec, model, p["lx"], p["nx"], p["ny"])
    for fname, text in (("spectrum.0", s), ("Xspectrum.0", xs), ("Yspectrum.0", ys)):
        assert open(os.path.join(tmp_path, "spectra", fname)).read() == text, fname
