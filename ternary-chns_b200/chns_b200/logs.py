"""The reference's diagnostic log files, written from the device diagnostics.

main.c's loop (main.c:216-226) calls free_energy(), kinetic_energy(), perimeter()
and spectrum() and each appends to its own text file; this module writes the same
files with the same printf formats, so the reference's post-processing reads them
unchanged:

  data/free_en_t.dat   "%lf \\t %.12lf \\t %.12lf"            t, E_bulk, E_grad (free_energy.c:149)
  data/ken_t.dat       "%lf \\t %.12lf[ \\t %.12lf ...]"       t, <|u|^2/2>, phase means (kinetic_energy.c:109-141)
  data/gamma.dat       "%g \\t %g \\t %g \\t %g"               t, Sp_0, Sp_t, def (perimeter.c:123; ternary
                                                           gamma1.dat / gamma2.dat, perimeter.c:264-265)
  spectra/spectrum.<i> "%.5e \\t %.12e ..."                  k, ek, ensk[, sph | sph1, sph2, sp12] (spectrum.c:150-165)
  spectra/Xspectrum.<i>, Yspectrum.<i>  "%d \\t %.12e"       (spectrum.c:168-187)

Python's %-formatting ignores the 'l' length modifier and rounds like printf.
"""
from __future__ import annotations

import math
import os


def free_energy_line(t: float, fe) -> str:
    return "%lf \t %.12lf \t %.12lf\n" % (t, fe[0], fe[1])


def kinetic_energy_line(t: float, model: int, ke) -> str:
    if model == 1:
        return "%lf \t %.12lf \t %.12lf\n" % (t, ke[0], ke[1])
    if model == 2:
        return "%lf \t %.12lf \t %.12lf \t %.12lf\n" % (t, ke[0], ke[1], ke[2])
    return "%lf \t %.12lf\n" % (t, ke[0])


def perimeter_line(t: float, per: dict) -> str:
    return "%g \t %g \t %g \t %g\n" % (t, per["sp_0"], per["sp_t"], per["def"])


def spectrum_text(spec: dict, model: int, lx: float, nx: int, ny: int, ly: float | None = None):
    """(spectrum, Xspectrum, Yspectrum) file contents of one spectrum() call."""
    ly = lx if ly is None else ly
    ek, ensk = spec["ek"], spec["ensk"]
    lines = []
    for ik in range(1, len(ek)):
        k = ik * (2 * math.pi / lx)
        if model == 1:
            lines.append("%.5e \t %.12e \t %.12e \t %.12e\n" % (k, ek[ik], ensk[ik], spec["sph"][ik]))
        elif model == 2:
            lines.append("%.5e \t %.12e \t %.12e \t %.12e \t %.12e \t %.12e\n"
                         % (k, ek[ik], ensk[ik], spec["sph1"][ik], spec["sph2"][ik], spec["sp12"][ik]))
        else:
            lines.append("%.5e \t %.12e \t %.12e\n" % (k, ek[ik], ensk[ik]))
    kxm = int(round(abs((nx / 2.0) * (2 * math.pi / lx))))  # main.c:57-63
    kym = int(round(abs((ny / 2.0) * (2 * math.pi / ly))))
    xs = "".join("%d \t %.12e\n" % (i, spec["ekx"][i]) for i in range(1, kxm))
    ys = "".join("%d \t %.12e\n" % (i, spec["eky"][i]) for i in range(1, kym))
    return "".join(lines), xs, ys


class Logs:
    """Appends the reference's per-step diagnostic lines for a Context under
    `directory` (data/, spectra/ are created)."""

    def __init__(self, ctx, directory: str):
        self.ctx = ctx
        self.dir = directory
        self.ifile = 0
        os.makedirs(os.path.join(directory, "data"), exist_ok=True)
        os.makedirs(os.path.join(directory, "spectra"), exist_ok=True)

    def _append(self, name: str, text: str):
        with open(os.path.join(self.dir, "data", name), "a") as f:
            f.write(text)

    def record(self, t: float, spectra: bool = True):
        """One iteration's diagnostics at time t, in main.c's order."""
        c = self.ctx
        fe, ke, rc = c.diagnostics()
        if c.model >= 1:
            self._append("free_en_t.dat", free_energy_line(t, fe))
        self._append("ken_t.dat", kinetic_energy_line(t, c.model, ke))
        if c.model >= 1:
            per = c.perimeter()
            if c.model == 1:
                self._append("gamma.dat", perimeter_line(t, per[0]))
            else:
                self._append("gamma1.dat", perimeter_line(t, per[0]))
                self._append("gamma2.dat", perimeter_line(t, per[1]))
        if spectra:
            p = c.params
            s, xs, ys = spectrum_text(c.spectrum(), c.model, p.get("lx", 2 * math.pi), c.nx, c.ny, p.get("ly"))
            for name, text in (("spectrum", s), ("Xspectrum", xs), ("Yspectrum", ys)):
                with open(os.path.join(self.dir, "spectra", f"{name}.{self.ifile}"), "w") as f:
                    f.write(text)
            self.ifile += 1
        return rc
