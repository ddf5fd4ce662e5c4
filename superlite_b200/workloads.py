"""Seeded synthetic inputs for SuperLite's per-timestep hot path.

No public dataset is involved: every array here is generated from a numpy
``default_rng(seed)`` with the shapes, sizes and value distributions of the
five benchmark configurations of the hot path:

1. 64-shell homologous ejecta (v in [0, 1.5e9] cm/s, broken power-law density,
   1 Msun, T ~ U(6000, 14000) K), analytic grey opacity
   kappa = 0.1 (rho/1e-13) (T/1e4)^-1.5 cm^2/g, 100 log groups 1000-32000 A,
   1e6 particles, 20 snapshots log-spaced in t = 1..30 d.
2. 256 shells, 2000 log groups, C/O/Ne/Mg/Si/S/Ca/Fe/Co/Ni Dirichlet mass
   fractions, 5e5 synthetic lines, Saha-Boltzmann ground-state populations.
3. The config-2 opacities driving a 5e7-particle IMC/DDMC timestep.
4. 128 independent models with 50..400 shells and 1e5..1e7 particles.
5. 4096 shells x 10000 groups x 2e6 lines.

Array layouts follow the reference's Fortran module arrays (column-major):
``cap`` is (ng, ncell) -> numpy shape (ncell, ng), group fastest.

The atomic data tables (Verner bound-free fits, Sutherland free-free Gaunt
factors) are synthetic tables of the reference's shapes (bfxsmod.f:14,
ffxsmod.f:18-20) unless ``load_verner``/``load_sutherland`` are given the
reference's data files.  The ionisation energies below are textbook values
(eV) for stages I-IV, used only to make plausible populations.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

# physconstmod.f:11-51
PC_C = 2.997924562e10
PC_KB = 1.3806505e-16
PC_H = 6.6260693e-27
PC_ME = 9.1093826e-28
PC_E = 4.80325e-10
PC_AMU = 1.66053886e-24
PC_EV = 1.60217653e-12
PC_MSUN = 1.989e33
PC_DAY = 86400.0
PC_PI = 3.1415926535897932385

NELEM = 30
# element numbers of the config-2 composition
ELEMENTS = (6, 8, 10, 12, 14, 16, 20, 26, 27, 28)
# atomic masses (amu) of the elements above
ELEM_MASS = {6: 12.011, 8: 15.999, 10: 20.180, 12: 24.305, 14: 28.086, 16: 32.06,
             20: 40.078, 26: 55.845, 27: 58.933, 28: 58.693}
# ionisation energies (eV) of stages I..IV
ION_ENERGY = {
    6: (11.260, 24.383, 47.888, 64.494),
    8: (13.618, 35.121, 54.936, 77.414),
    10: (21.565, 40.963, 63.423, 97.190),
    12: (7.646, 15.035, 80.144, 109.265),
    14: (8.152, 16.346, 33.493, 45.142),
    16: (10.360, 23.338, 34.790, 47.222),
    20: (6.113, 11.872, 50.913, 67.273),
    26: (7.902, 16.199, 30.651, 54.910),
    27: (7.881, 17.084, 33.500, 51.270),
    28: (7.640, 18.169, 35.187, 54.920),
}
NSTAGE = 4          # ion stages with bound electrons carried per element (I-IV)
ION_NI = 5          # ion_el(iz)%ni: stages I..V, the last one carries no lines


@dataclasses.dataclass
class Grid:
    """1-D spherical homologous grid (grd_xarr, grd_vxarr, grd_vol, grd_divv)."""
    nx: int
    t: float
    xarr: np.ndarray
    vxarr: np.ndarray
    vol: np.ndarray
    divv: np.ndarray


@dataclasses.dataclass
class Groups:
    ng: int
    wl: np.ndarray      # grp_wl (ng+1) [cm]
    wlinv: np.ndarray   # grp_wlinv (ng+1)

    @property
    def nep(self) -> int:          # gridmod.f:121
        return int(round(math.sqrt(float(self.ng))))

    @property
    def nepg(self) -> int:         # gridmod.f:122
        return int(math.ceil(self.ng / (self.nep + 1.0)))


@dataclasses.dataclass
class Gas:
    """Per-shell gas state (gasmod.f) for the physical opacity."""
    temp: np.ndarray
    mass: np.ndarray
    rho: np.ndarray
    natom: np.ndarray
    nelec: np.ndarray
    natomfr: np.ndarray        # (ncell, 0:nelem) -> shape (ncell, nelem+1)
    massfr: np.ndarray         # (ncell, nelem)
    ion_ni: np.ndarray         # (nelem,) int32
    oc: np.ndarray             # (nelem, nstage, ncell) ion_grndlev%oc
    ginv: np.ndarray           # (nelem, nstage, ncell) ion_grndlev%ginv


BBXS_DTYPE = np.dtype([("wl0", "<f4"), ("gxs", "<f4"), ("chilw", "<f4"),
                       ("iz", "<i2"), ("ii", "<i2")])  # bbxsmod.f:27-34, 16 bytes


def group_grid(ng: int, wlmin: float = 1000e-8, wlmax: float = 32000e-8) -> Groups:
    """Log-spaced group edges, groupmod.f:45-47."""
    ig = np.arange(1, ng + 2, dtype=np.float64)
    wl = wlmin * (wlmax / wlmin) ** ((ig - 1.0) / ng)
    return Groups(ng, wl, 1.0 / wl)


def homologous_grid(nx: int, t: float, vmax: float = 1.5e9) -> Grid:
    """Linear velocity edges 0..vmax at time t (grid_setup.f:46-52, grid_volume.f:82-87)."""
    vx = np.linspace(0.0, vmax, nx + 1)
    x = vx * t
    vol = (x[1:] ** 3 - x[:-1] ** 3) * 2.0 * (2.0 * PC_PI) / 3.0
    divv = 2 * (vx[1:] + vx[:-1]) / (x[1:] + x[:-1]) + (vx[1:] - vx[:-1]) / (x[1:] - x[:-1])
    return Grid(nx, t, x, vx, vol, divv)


def broken_powerlaw_rho(grid: Grid, vb: float = 5e8, mtot: float = PC_MSUN):
    """rho ~ v^-1 (v < vb), v^-7 (v >= vb) at cell centres, normalised to mtot."""
    vc = 0.5 * (grid.vxarr[1:] + grid.vxarr[:-1])
    shape = np.where(vc < vb, (vc / vb) ** -1.0, (vc / vb) ** -7.0)
    mass = shape * grid.vol
    mass *= mtot / mass.sum()
    return mass / grid.vol, mass


def snapshot_times(n: int = 20, t0_days: float = 1.0, t1_days: float = 30.0) -> np.ndarray:
    return np.geomspace(t0_days, t1_days, n) * PC_DAY


# ---------------------------------------------------------------- atomic data
def synthetic_verner(seed: int = 7):
    """bf_ph1(6,7,30,30) and bf_ph2(7,30,30) shaped tables with Verner-like fits.

    ph1(:,is,nz,ne) = (E_th, E_0, sigma_0, y_a, P, y_w) per shell; ph2(:,nz,ne) =
    (E_0, sigma_0, y_a, P, y_w, y_0, y_1).  Thresholds follow a screened
    hydrogenic ladder so inner shells lie above outer ones.
    Returned in Fortran order, flattened to 1-D float32 arrays.
    """
    rng = np.random.default_rng(seed)
    ph1 = np.zeros((30, 30, 7, 6), dtype=np.float32)   # (ne, nz, is, k) C-order
    ph2 = np.zeros((30, 30, 7), dtype=np.float32)      # (ne, nz, k)
    nshell = [1, 1, 2, 2, 3, 3, 3, 3, 3, 3, 4, 4, 5, 5, 5, 5, 5, 5, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 7, 7]
    nprin = [1, 2, 2, 3, 3, 3, 4]
    for nz in range(1, 31):
        for ne in range(1, nz + 1):
            nout = nshell[ne - 1]
            if nz > 18 and (nz == ne or (nz == ne + 1 and nz in (20, 21, 22, 25, 26))):
                nout = 7  # bfxsmod.f:225-231
            for is_ in range(1, nout + 1):
                zeff = max(1.0, nz - 0.85 * (ne - 1) * (is_ / max(nout, 1)))
                eth = 13.6 * zeff ** 2 / nprin[is_ - 1] ** 2 * rng.uniform(0.8, 1.2)
                ph1[ne - 1, nz - 1, is_ - 1] = (eth, eth * rng.uniform(0.3, 3.0),
                                                10 ** rng.uniform(0.5, 4.0), rng.uniform(1.0, 60.0),
                                                rng.uniform(2.5, 14.0), rng.uniform(0.0, 0.6))
            e0 = ph1[ne - 1, nz - 1, nout - 1, 0]
            ph2[ne - 1, nz - 1] = (e0 * rng.uniform(0.3, 2.0), 10 ** rng.uniform(0.5, 4.0),
                                   rng.uniform(1.0, 60.0), rng.uniform(2.5, 14.0),
                                   rng.uniform(0.0, 0.6), rng.uniform(0.0, 1.0), rng.uniform(0.0, 1.0))
    return np.ascontiguousarray(ph1).ravel(), np.ascontiguousarray(ph2).ravel()


def load_verner(path: str):
    """Read a data.bf_verner file (bfxsmod.f:144-180) into the two flat tables."""
    with open(path) as f:
        lines = f.read().split("\n")
    vals1, vals2, part = [], [], 0
    for ln in lines:
        s = ln.strip()
        if not s:
            continue
        if s.startswith("#"):
            part += 1
            continue
        (vals1 if part <= 2 else vals2).extend(float(v) for v in s.split())
    ph1d = np.array(vals1, dtype=np.float32).reshape(1699, 9)
    ph2d = np.array(vals2, dtype=np.float32).reshape(465, 9)
    ph1 = np.zeros((30, 30, 7, 6), dtype=np.float32)
    ph2 = np.zeros((30, 30, 7), dtype=np.float32)
    for r in ph1d:
        ns, ne, nz = int(round(r[0])), int(round(r[1])), int(round(r[2]))
        ph1[ne - 1, nz - 1, ns - 1] = r[3:]
    for r in ph2d:
        ne, nz = int(round(r[0])), int(round(r[1]))
        ph2[ne - 1, nz - 1] = r[2:]
    return np.ascontiguousarray(ph1).ravel(), np.ascontiguousarray(ph2).ravel()


def synthetic_gaunt() -> np.ndarray:
    """ff_gff(81,41) shaped table: smooth free-free Gaunt factors on the
    reference's grid (log10 u = -4..4 step 0.1, log10 gamma^2 = -4..4 step 0.2)."""
    lu = -4.0 + 0.1 * np.arange(81)
    lg = -4.0 + 0.2 * np.arange(41)
    U, G = np.meshgrid(lu, lg, indexing="ij")
    gff = 1.0 + 0.55 * np.log1p(np.exp(-1.2 * U)) * (1.0 + 0.1 * np.tanh(G)) + 0.05 * np.sin(U + G)
    return np.asfortranarray(gff).ravel(order="F")


def load_sutherland(path: str) -> np.ndarray:
    """Read data.ff_sutherland (ffxsmod.f:345-371): third column, u fastest."""
    with open(path) as f:
        rows = f.read().split("\n")[5:]
    vals = np.array([float(v) for r in rows for v in r.split()], dtype=np.float64)
    return vals.reshape(41, 81, 3)[:, :, 2].ravel()  # Fortran (81,41) flattened


# ------------------------------------------------------------- populations
@dataclasses.dataclass
class IonTable:
    """Ion data of ions_read_data (ionsmod.f:652-829) in the layouts of
    slg_set_ions: per element iz (1..nelem) ni stages including the bare ion;
    e (nelem, nstage) ionisation energy of stage ii -> ii+1 [erg]; levels
    glev/elev (nelem, nstage, nlev) [elev in erg], nlevel (nelem, nstage)."""
    ni: np.ndarray
    e: np.ndarray
    nlevel: np.ndarray
    glev: np.ndarray
    elev: np.ndarray

    @property
    def nelem(self) -> int:
        return len(self.ni)

    @property
    def nstage(self) -> int:
        return self.e.shape[1]

    @property
    def g1(self) -> np.ndarray:
        return self.glev[:, :, 0]


def ion_table(seed: int = 7, nlev: int = 6) -> IonTable:
    """Synthetic ion data for all NELEM elements with ION_NI stages: the
    energies of ION_ENERGY for the config-2 elements (seeded hydrogen-like
    values for the others), a ground level with a small integer weight and
    nlev-1 excited levels below the ionisation energy; the bare ion has one
    level of weight 1."""
    rng = np.random.default_rng(seed)
    ns = ION_NI
    ni = np.full(NELEM, ns, dtype=np.int32)
    e = np.zeros((NELEM, ns))
    nlevel = np.zeros((NELEM, ns), dtype=np.int32)
    glev = np.zeros((NELEM, ns, nlev))
    elev = np.zeros((NELEM, ns, nlev))
    for iz in range(1, NELEM + 1):
        if iz in ION_ENERGY:
            ev = np.array(ION_ENERGY[iz])
        else:
            ev = np.sort(rng.uniform(6.0, 14.0) * np.array([1.0, 2.1, 3.4, 4.9]) * rng.uniform(0.9, 1.1, 4))
        e[iz - 1, :ns - 1] = ev * PC_EV
        for ii in range(ns - 1):
            nlevel[iz - 1, ii] = nlev
            glev[iz - 1, ii, 0] = float(rng.choice([1, 2, 3, 4, 5, 6, 9]))
            glev[iz - 1, ii, 1:] = rng.integers(1, 16, nlev - 1).astype(np.float64)
            elev[iz - 1, ii, 1:] = np.sort(rng.uniform(0.05, 0.8, nlev - 1)) * ev[ii] * PC_EV
        nlevel[iz - 1, ns - 1] = 1
        glev[iz - 1, ns - 1, 0] = 1.0
    return IonTable(ni, e, nlevel, glev, elev)


@dataclasses.dataclass
class AtomicData:
    """The reference's atomic data (Data/data.bf_verner, data.ff_sutherland,
    data.ion and a subset of Atoms/data.atom.*), as parsed into an npz file by
    tests/golden/make_atomic_data.py."""
    bf_ph1: np.ndarray      # flat float32, bf_ph1(6,7,30,30)
    bf_ph2: np.ndarray      # flat float32, bf_ph2(7,30,30)
    ff_gff: np.ndarray      # flat float64, ff_gff(81,41)
    ion: "IonTable"
    lines: np.ndarray       # BBXS_DTYPE, sorted by wl0

    @property
    def tables(self):
        return self.bf_ph1, self.bf_ph2, self.ff_gff


def ion_table_from_levels(icod, ip_cm, nlev, chi_cm, g, nelem: int = NELEM) -> "IonTable":
    """ions_read_data (ionsmod.f:652-829) on parsed data.ion records: stage ii of
    element iz (icod = 100 iz + ii - 1) gets e = h c IP and levels (h c chi, g);
    ni is the first stage without levels (ionsmod.f:787-794), which becomes the
    bare ion with one level of weight 1 (:797-806)."""
    hc = PC_H * PC_C
    starts = np.concatenate([[0], np.cumsum(nlev)])
    per = {}
    for k, code in enumerate(icod):
        iz, ii = int(code) // 100, int(code) % 100 + 1
        if iz <= nelem:
            per[(iz, ii)] = (float(ip_cm[k]), chi_cm[starts[k]:starts[k + 1]], g[starts[k]:starts[k + 1]])
    ni = np.zeros(nelem, dtype=np.int32)
    for iz in range(1, nelem + 1):
        l = 1
        while l <= iz + 1 and (iz, l) in per and len(per[(iz, l)][1]) > 0:
            l += 1
        ni[iz - 1] = l
    ns = int(ni.max())
    nl = max(len(v[1]) for v in per.values())
    e = np.zeros((nelem, ns))
    nlevel = np.zeros((nelem, ns), dtype=np.int32)
    glev = np.zeros((nelem, ns, nl))
    elev = np.zeros((nelem, ns, nl))
    for iz in range(1, nelem + 1):
        for ii in range(1, int(ni[iz - 1])):
            p, c, gg = per[(iz, ii)]
            e[iz - 1, ii - 1] = hc * p
            nlevel[iz - 1, ii - 1] = len(c)
            glev[iz - 1, ii - 1, :len(c)] = gg
            elev[iz - 1, ii - 1, :len(c)] = hc * np.asarray(c)
        top = int(ni[iz - 1]) - 1
        nlevel[iz - 1, top] = 1
        glev[iz - 1, top, 0] = 1.0
    return IonTable(ni, e, nlevel, glev, elev)


def load_atomic_data(path: str) -> AtomicData:
    """Read the npz written by tests/golden/make_atomic_data.py."""
    d = np.load(path)
    ion = ion_table_from_levels(d["ion_icod"], d["ion_ip_cm"], d["ion_nlev"], d["lev_chi_cm"],
                                d["lev_g"].astype(np.float64))
    return AtomicData(d["bf_ph1"], d["bf_ph2"], d["ff_gff"], ion, d["lines"])


def composition_state(rho: np.ndarray, massfr: np.ndarray, vol: np.ndarray):
    """massfr2natomfr (GAS/gas_setup.f:101-160) for given mass fractions:
    gas_mass = rho vol, X renormalised to sum 1, number fractions
    natomfr(0:nelem) ~ X_z / A_z normalised to 1, gas_natom = mass sum(X_z/A_z) / amu.  massfr is (ncell, NELEM) over
    elements 1..NELEM; elements without a mass in ELEM_MASS take 2 z amu."""
    A = np.array([ELEM_MASS.get(z, 2.0 * z) for z in range(1, NELEM + 1)])
    mass = rho * vol
    y = (massfr / massfr.sum(axis=1, keepdims=True)) / A
    s = y.sum(axis=1)
    natomfr = np.zeros((len(rho), NELEM + 1))
    natomfr[:, 1:] = y / s[:, None]
    natom = mass * s / PC_AMU
    return mass, natom, natomfr


def _saha_cell(temp: float, ndens: float, natomfr_el: np.ndarray):
    """Synthetic two-level Saha balance: returns (nelec per atom, stage fractions)."""
    kt = PC_KB * temp
    sahac = (2 * PC_PI * PC_ME * PC_KB * temp / PC_H ** 2) ** 1.5
    chi = np.array([ION_ENERGY[z] for z in ELEMENTS]) * PC_EV   # (nel, 4)

    def fractions(ne_dens):
        # ratio n_{j+1}/n_j with equal ground-state weights
        lr = np.log(2.0 * sahac / ne_dens) - chi / kt               # (nel, 4)
        lcum = np.concatenate([np.zeros((len(ELEMENTS), 1)), np.cumsum(lr, axis=1)], axis=1)
        lcum -= lcum.max(axis=1, keepdims=True)
        f = np.exp(lcum)
        return f / f.sum(axis=1, keepdims=True)                     # (nel, 5)

    lo, hi = math.log(1e-8 * ndens), math.log(4.0 * ndens)
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        f = fractions(math.exp(mid))
        ne_pred = ndens * float((natomfr_el[:, None] * f * np.arange(5)).sum())
        if ne_pred > math.exp(mid):
            lo = mid
        else:
            hi = mid
    ne_dens = math.exp(0.5 * (lo + hi))
    return ne_dens / ndens, fractions(ne_dens)


def make_gas(grid: Grid, rng: np.random.Generator, temp: Optional[np.ndarray] = None,
             mtot: float = PC_MSUN) -> Gas:
    """Dirichlet(1) mass fractions per shell, number fractions, Saha populations."""
    nc = grid.nx
    rho, mass = broken_powerlaw_rho(grid, mtot=mtot)
    if temp is None:
        temp = rng.uniform(6000.0, 14000.0, nc)
    X = rng.dirichlet(np.ones(len(ELEMENTS)), size=nc)                # (nc, nel)
    A = np.array([ELEM_MASS[z] for z in ELEMENTS])
    nfr = X / A
    mu_inv = nfr.sum(axis=1)
    natom = mass * mu_inv / PC_AMU
    natomfr = np.zeros((nc, NELEM + 1))
    massfr = np.zeros((nc, NELEM))
    ion_ni = np.full(NELEM, ION_NI, dtype=np.int32)
    oc = np.zeros((NELEM, NSTAGE, nc))
    ginv = np.ones((NELEM, NSTAGE, nc))
    nelec = np.zeros(nc)
    for i in range(nc):
        fr = nfr[i] / mu_inv[i]
        ndens = natom[i] / grid.vol[i]
        ne_per_atom, f = _saha_cell(float(temp[i]), ndens, fr)
        nelec[i] = ne_per_atom
        for k, z in enumerate(ELEMENTS):
            natomfr[i, z] = fr[k]
            massfr[i, z - 1] = X[i, k]
            # oc = natom*natomfr*g1*n/(q*vol) with q = g1 (two-level)
            oc[z - 1, :, i] = natom[i] * fr[k] * f[k, :NSTAGE] / grid.vol[i]
    return Gas(temp, mass, rho, natom, nelec, natomfr, massfr, ion_ni, oc, ginv)


def make_lines(nline: int, rng: np.random.Generator, wlmin_ang: float = 1000.0,
               wlmax_ang: float = 32000.0) -> np.ndarray:
    """Synthetic line list packed like bb_xs (read_bbxs_data.f:60-73), sorted by wl0."""
    fconst = PC_PI * PC_E ** 2 / (PC_ME * PC_C)
    wl0 = np.exp(rng.uniform(math.log(wlmin_ang), math.log(wlmax_ang), nline))
    loggf = rng.normal(-2.0, 1.5, nline)
    elow_ev = rng.uniform(0.0, 10.0, nline)
    iz = np.array(ELEMENTS, dtype=np.int16)[rng.integers(0, len(ELEMENTS), nline)]
    ii = rng.integers(1, NSTAGE + 1, nline).astype(np.int16)
    bb = np.zeros(nline, dtype=BBXS_DTYPE)
    bb["wl0"] = wl0.astype(np.float32)
    bb["gxs"] = (np.float32(fconst) * np.float32(10.0) ** loggf.astype(np.float32)).astype(np.float32)
    bb["chilw"] = (elow_ev * PC_EV / (PC_H * PC_C)).astype(np.float32)
    bb["iz"] = iz
    bb["ii"] = ii
    order = np.argsort(bb["wl0"], kind="stable")
    return bb[order]


# ------------------------------------------------------------- opacity cases
@dataclasses.dataclass
class OpacityCase:
    grid: Grid
    groups: Groups
    gas: Gas
    lines: np.ndarray
    bf_ph1: np.ndarray
    bf_ph2: np.ndarray
    ff_gff: np.ndarray


def opacity_case(ncell: int = 256, ng: int = 2000, nline: int = 500_000, seed: int = 2,
                 t_days: float = 10.0, tables=None) -> OpacityCase:
    """Config 2 (defaults) or a scaled variant: physical LTE opacity inputs."""
    rng = np.random.default_rng(seed)
    grid = homologous_grid(ncell, t_days * PC_DAY)
    groups = group_grid(ng)
    gas = make_gas(grid, rng)
    lines = make_lines(nline, rng)
    if tables is None:
        ph1, ph2 = synthetic_verner()
        gff = synthetic_gaunt()
    else:
        ph1, ph2, gff = tables
    return OpacityCase(grid, groups, gas, lines, ph1, ph2, gff)


@dataclasses.dataclass
class ModelBatch:
    """Independent ejecta models laid out for slg_set_models: per-model grids
    and gas, and the concatenations the library reads (edges model after
    model, per-cell arrays over all cells)."""
    models: list            # one OpacityCase per model (shared groups, lines, tables)
    nx: np.ndarray          # shells per model (int32)
    npart: np.ndarray       # particle slots per model (int64)
    t_days: np.ndarray
    xarr: np.ndarray
    vxarr: np.ndarray
    vol: np.ndarray
    divv: np.ndarray
    gas: Gas                # all cells, model order

    @property
    def groups(self) -> Groups:
        return self.models[0].groups

    @property
    def lines(self) -> np.ndarray:
        return self.models[0].lines


def concat_gas(gases) -> Gas:
    cat0 = lambda k: np.concatenate([getattr(g, k) for g in gases], axis=0)
    cat2 = lambda k: np.concatenate([getattr(g, k) for g in gases], axis=2)
    return Gas(cat0("temp"), cat0("mass"), cat0("rho"), cat0("natom"), cat0("nelec"), cat0("natomfr"),
               cat0("massfr"), gases[0].ion_ni, cat2("oc"), cat2("ginv"))


def model_batch(nmodel: int = 128, seed: int = 4, ng: int = 2000, nline: int = 500_000,
                nx_range=(50, 400), npart_range=(1e5, 1e7), t_range_days=(1.0, 30.0),
                nx=None, npart=None) -> ModelBatch:
    """Batched workload: shells ~ U{nx_range}, particle budgets log-uniform in
    npart_range, snapshot times log-uniform in t_range_days, and per model
    seeded T (U(6000, 14000) K), broken-power-law rho (1 Msun) and
    Dirichlet(1) composition as in opacity_case.  Groups, the line list and
    the bf/ff tables are shared by every model."""
    rng = np.random.default_rng(seed)
    nxs = (rng.integers(nx_range[0], nx_range[1] + 1, nmodel) if nx is None
           else np.asarray(nx)).astype(np.int32)
    nps = (np.exp(rng.uniform(math.log(npart_range[0]), math.log(npart_range[1]), nmodel)).astype(np.int64)
           if npart is None else np.asarray(npart, dtype=np.int64))
    ts = np.exp(rng.uniform(math.log(t_range_days[0]), math.log(t_range_days[1]), nmodel))
    groups = group_grid(ng)
    lines = make_lines(nline, rng)
    ph1, ph2 = synthetic_verner()
    gff = synthetic_gaunt()
    models = []
    for m in range(nmodel):
        mr = np.random.default_rng([seed, m])
        grid = homologous_grid(int(nxs[m]), float(ts[m]) * PC_DAY)
        models.append(OpacityCase(grid, groups, make_gas(grid, mr), lines, ph1, ph2, gff))
    cat = lambda k: np.concatenate([getattr(c.grid, k) for c in models])
    return ModelBatch(models, nxs, nps, ts, cat("xarr"), cat("vxarr"), cat("vol"), cat("divv"),
                      concat_gas([c.gas for c in models]))


@dataclasses.dataclass
class AnalyticBatch:
    """Independent ejecta models with the CPU-runnable case's physics (analytic grey
    opacity, so no composition enters), laid out for slg_set_models."""
    nx: np.ndarray          # shells per model (int32)
    npart: np.ndarray       # particle slots per model (int64)
    t_days: np.ndarray
    groups: Groups
    xarr: np.ndarray        # each model's nx+1 edges, model after model
    vxarr: np.ndarray
    vol: np.ndarray         # per cell, model order
    divv: np.ndarray
    temp: np.ndarray
    rho: np.ndarray


def analytic_batch(nmodel: int = 128, seed: int = 4, ng: int = 100, nx_range=(50, 400),
                   npart_range=(1e5, 1e7), t_range_days=(1.0, 30.0), nx=None, npart=None) -> AnalyticBatch:
    """The batched workload: nmodel models with shells ~ U{nx_range},
    particle budgets log-uniform in npart_range and snapshot times
    log-uniform in t_range_days; per model (seed [seed, m]) T ~ U(6000, 14000)
    K and a 1 Msun broken power-law density; 100 log groups."""
    rng = np.random.default_rng(seed)
    nxs = (rng.integers(nx_range[0], nx_range[1] + 1, nmodel) if nx is None
           else np.asarray(nx)).astype(np.int32)
    nps = (np.exp(rng.uniform(math.log(npart_range[0]), math.log(npart_range[1]), nmodel)).astype(np.int64)
           if npart is None else np.asarray(npart, dtype=np.int64))
    ts = np.exp(rng.uniform(math.log(t_range_days[0]), math.log(t_range_days[1]), len(nxs)))
    grids, temps, rhos = [], [], []
    for m in range(len(nxs)):
        mr = np.random.default_rng([seed, m])
        g = homologous_grid(int(nxs[m]), float(ts[m]) * PC_DAY)
        rho, _ = broken_powerlaw_rho(g)
        grids.append(g)
        temps.append(mr.uniform(6000.0, 14000.0, int(nxs[m])))
        rhos.append(rho)
    cat = lambda k: np.concatenate([getattr(g, k) for g in grids])
    return AnalyticBatch(nxs, nps, ts, group_grid(ng), cat("xarr"), cat("vxarr"), cat("vol"), cat("divv"),
                         np.concatenate(temps), np.concatenate(rhos))


def analytic_grey(grid: Grid, temp: np.ndarray, rho: np.ndarray, ng: int):
    """Config-1 opacity source: in_opacanaltype='grey', capcoef=1e18,
    captpwr=-1.5, caprpwr=2 (analytic_opacity.f90:38-43); sigma = 0."""
    cap = (1e18 * temp ** -1.5 * rho ** 2.0)
    return np.zeros_like(temp), np.repeat(cap.astype(np.float32)[:, None], ng, axis=1)


@dataclasses.dataclass
class TransportParams:
    tauddmc: float = 5.0       # inputparmod.f:54
    taulump: float = 10.0      # inputparmod.f:55
    puretran: bool = False
    noampfact: bool = True     # inputparmod.f:57
    errorfatal: bool = True
    thm_aniso: bool = False
    dogrdtally: bool = False
    max_steps: int = 10_000_000


# ------------------------------------------------------------- source particles
HCK = PC_H * PC_C / PC_KB
FTPI4 = 15.0 / PC_PI ** 4


def planck_group_weights(tempinv: float, wlinv: np.ndarray) -> np.ndarray:
    """specintv mode 0 (groupmod.f:189-198) in numpy."""
    x = HCK * tempinv * wlinv
    xm = 0.5 * (x[1:] + x[:-1])
    f = np.where(xm >= 300.0, 300.0 ** 3 / np.expm1(300.0), xm ** 3 / np.expm1(np.minimum(xm, 300.0)))
    return FTPI4 * np.abs(x[1:] - x[:-1]) * f


def source_numbers(emit: np.ndarray, src_ns: int) -> np.ndarray:
    """sourcenumbers.f90:3-94 for one rank without a surface source."""
    nx = len(emit)
    etot = emit.sum()
    nvol = np.zeros(nx, dtype=np.int64)
    edone, ndone = 0.0, 0
    invn, einv = 1.0 / src_ns, 1.0 / etot
    for l in range(nx):
        en = emit[l]
        if en == 0.0:
            continue
        n = max(1, int(en * src_ns * einv))
        if edone * einv > ndone * invn:
            n += 1
        nvol[l] = n
        edone += en
        ndone += n
    ncactive = int((emit > 0).sum())
    nextra = src_ns - int(nvol.sum())
    nsmean = src_ns // ncactive
    while nextra != 0:
        for l in range(nx):
            if nextra == 0:
                break
            if nvol[l] < nsmean:
                continue
            s = 1 if nextra > 0 else -1
            nvol[l] += s
            nextra -= s
    return nvol


def source_particles(grid: Grid, groups: Groups, radtemp: np.ndarray, L_bol: float, npart: int,
                     seed: int = 0):
    """Thermal "surface" source in every shell with the distributions of
    sourceenergy.f90, interior_source.f90 and source_transformdirection.f90
    (vectorised numpy, own random stream).  Returns (packets, isvacant)."""
    from .api import PACKET_DTYPE
    rng = np.random.default_rng(seed)
    x, vx = grid.xarr, grid.vxarr
    rcell = 0.5 * (x[1:] + x[:-1])
    emit = PC_PI * PC_C * rcell ** 2 * 7.5657e-15 * radtemp ** 4
    emit = emit / emit.sum() * L_bol
    nvol = source_numbers(emit, npart)
    buf = np.zeros((npart, 8))  # x, y, z, mu, om, e, e0, wl
    k = 0
    nx = grid.nx
    for i in range(nx):
        n = int(nvol[i])
        if n == 0:
            continue
        w = planck_group_weights(1.0 / radtemp[i], groups.wlinv)
        cdf = np.cumsum(w / w.sum())
        r = rng.random(n)
        ig = np.minimum(np.searchsorted(cdf, r, side="right"), groups.ng - 1)
        r = rng.random(n)
        wl = 1.0 / ((1.0 - r) * groups.wlinv[ig] + r * groups.wlinv[ig + 1])
        mu = np.sqrt(rng.random(n))
        om = 2 * PC_PI * rng.random(n)
        uul = 0.5 * (emit[max(i - 1, 0)] + emit[i])
        uur = 0.5 * (emit[min(i + 1, nx - 1)] + emit[i])
        um = max(uul, uur)
        uul, uur = uul / um, uur / um
        x0 = np.empty(n)
        todo = np.arange(n)
        while len(todo):
            r1 = rng.random(len(todo))
            xs = (r1 * x[i + 1] ** 3 + (1 - r1) * x[i] ** 3) ** (1.0 / 3.0)
            r3 = (xs - x[i]) / (x[i + 1] - x[i])
            r3 = r3 * uur + (1 - r3) * uul
            acc = rng.random(len(todo)) <= r3
            x0[todo[acc]] = xs[acc]
            todo = todo[~acc]
        v = (vx[i] * (x[i + 1] - x0) + vx[i + 1] * (x0 - x[i])) / (x[i + 1] - x[i])
        mul = np.clip((mu + v / PC_C) / (1.0 + mu * v / PC_C), -1.0, 1.0)
        b = buf[k:k + n]
        b[:, 0], b[:, 1], b[:, 2], b[:, 3], b[:, 4] = x0, -1.0, 0.0, mul, om
        b[:, 5] = b[:, 6] = emit[i] / n
        b[:, 7] = wl
        k += n
    return buf.view(PACKET_DTYPE).reshape(npart), np.zeros(npart, dtype=np.int32)
