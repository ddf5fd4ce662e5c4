"""The reference's output files for the results of the hot path, so that the
C-ABI's luminosities and totals drop into SuperLite's existing
post-processing (e.g. Tools/sgfilter.py, which reads output.flx_luminos with
numpy.loadtxt and the wavelength edges from line 2 of output.flx_grid).

Formats follow OUTPUT/output_flux.f:16-68 and the output.tot_energy block of
OUTPUT/output_grid.f:55-64:

* output.flx_grid (written once): a "#" header with flx_ng, flx_nmu, flx_nom,
  then the edges flx_wl, flx_mu, flx_om, each as one row of 1pe12.4 fields;
* output.flx_luminos / output.flx_lumdev: per step one row of flx_ng 1pe12.4
  fields per (mu, om) bin, values not above 1e-99 written as 0 (the
  reference's merge(..., mask=x>1d-99), which keeps three-digit exponents out
  of the 12-character fields); output.flx_lumnum: the counts as i12;
* output.tot_energy: two "#" header lines, then per step eout, evelo, sflux,
  sthermal as 1pe12.4.

A file set is started (replaced) by the first write of a writer object and
appended to afterwards, as the reference's lfirst/fstat logic does.
"""
from __future__ import annotations

import os

import numpy as np


def _e12(values) -> str:
    """Fortran '1p,e12.4' fields: one digit before the point, 4 after."""
    return "".join(f"{float(v):12.4E}" for v in np.ravel(values))


def _i12(values) -> str:
    return "".join(f"{int(v):12d}" for v in np.ravel(values))


def _masked(a):
    a = np.asarray(a, dtype=np.float64)
    return np.where(a > 1e-99, a, 0.0)


class FluxOutput:
    """output_flux for one model: ``write(luminos, lumdev, lumnum)`` per step.

    luminos/lumdev/lumnum are (flx_ng,) for one (mu, om) bin, or
    (flx_nmu * flx_nom, flx_ng) with mu fastest (the reference's j, k loops)."""

    def __init__(self, directory: str, flx_wl, flx_mu=(-1.0, 1.0), flx_om=(0.0, 2.0 * np.pi)):
        self.dir = directory
        self.wl = np.asarray(flx_wl, dtype=np.float64)
        self.mu = np.asarray(flx_mu, dtype=np.float64)
        self.om = np.asarray(flx_om, dtype=np.float64)
        self.ng, self.nmu, self.nom = len(self.wl) - 1, len(self.mu) - 1, len(self.om) - 1
        self.first = True
        os.makedirs(directory, exist_ok=True)

    def _path(self, name):
        return os.path.join(self.dir, name)

    def write(self, luminos, lumdev, lumnum):
        rows = self.nmu * self.nom
        lum = np.asarray(luminos, dtype=np.float64).reshape(rows, self.ng)
        dev = np.asarray(lumdev, dtype=np.float64).reshape(rows, self.ng)
        num = np.asarray(lumnum).reshape(rows, self.ng)
        if self.first:
            with open(self._path("output.flx_grid"), "w") as f:
                f.write(f" #{self.ng:12d}{self.nmu:12d}{self.nom:12d}\n")
                f.write(_e12(self.wl) + "\n")
                f.write(_e12(self.mu) + "\n")
                f.write(_e12(self.om) + "\n")
        mode = "w" if self.first else "a"
        with open(self._path("output.flx_luminos"), mode) as f:
            for r in range(rows):
                f.write(_e12(_masked(lum[r])) + "\n")
        with open(self._path("output.flx_lumnum"), mode) as f:
            for r in range(rows):
                f.write(_i12(num[r]) + "\n")
        with open(self._path("output.flx_lumdev"), mode) as f:
            for r in range(rows):
                f.write(_e12(_masked(dev[r])) + "\n")
        self.first = False


class EnergyOutput:
    """output.tot_energy: eout, evelo, sflux, sthermal per step."""

    def __init__(self, directory: str):
        self.path = os.path.join(directory, "output.tot_energy")
        self.first = True
        os.makedirs(directory, exist_ok=True)

    def write(self, eout: float, evelo: float, sflux: float, sthermal: float):
        with open(self.path, "w" if self.first else "a") as f:
            if self.first:
                f.write("#    4\n")
                f.write("#" + "".join(f"{s:>12s}" for s in ("eout", "evelo", "sflux", "sthermal")) + "\n")
            f.write(" " + _e12([eout, evelo, sflux, sthermal]) + "\n")
        self.first = False


def model_flux_writers(directory: str, nmodel: int, flx_wl):
    """One FluxOutput per model of a batch (subdirectories model_0000, ...):
    row m of the batched slg_fluxtally result goes to writer m."""
    return [FluxOutput(os.path.join(directory, f"model_{m:04d}"), flx_wl) for m in range(nmodel)]
