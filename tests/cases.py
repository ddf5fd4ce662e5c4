"""Seeded parity cases shared by the GPU tests (small enough for the oracle)."""
import os

import numpy as np

from superlite_b200 import workloads as W


def opacity_case(ncell=64, ng=200, nline=20000, seed=11, t_days=10.0, ngs=1):
    return W.opacity_case(ncell=ncell, ng=ng, nline=nline, seed=seed, t_days=t_days)


def transport_case(oracle, t_days=5.0, nx=64, ng=100, npart=4000, seed=3, kind="grey", params=None,
                   L_bol=1e42):
    """Config-1 shaped snapshot: returns dict with grid, groups, tables, particles."""
    rng = np.random.default_rng(seed)
    grid = W.homologous_grid(nx, t_days * W.PC_DAY)
    groups = W.group_grid(ng)
    rho, mass = W.broken_powerlaw_rho(grid)
    temp = rng.uniform(6000.0, 14000.0, nx)
    if kind == "mono":  # group-dependent: ~70% of (shell, group) pairs optically thick at 6 d
        sig, cap = oracle.analytic_opacity(groups.wlinv, temp, rho, kind=2, capcoef=1e33)
    else:
        sig, cap = oracle.analytic_opacity(groups.wlinv, temp, rho, kind=1)
    if kind == "grey+sig":
        sig = 0.3 * cap[:, 0].astype(np.float64)
    tinv = 1.0 / temp
    capgrey = oracle.planckmean(groups.wlinv, temp, cap)
    params = params or W.TransportParams()
    ol = oracle.leakage_opacity11(grid, groups.wlinv, tinv, sig, cap, tauddmc=params.tauddmc,
                                  taulump=params.taulump)
    ep = oracle.emission_probability(groups.wlinv, tinv, cap, capgrey, groups.nep, groups.nepg)
    prt, isv, emit, nvol, tot = oracle.make_source_particles(grid, groups, temp, L_bol, npart)
    tables = dict(tempinv=tinv, sig=sig, capgrey=capgrey, emitprob=ep, opaclump=ol, cap=cap)
    return dict(grid=grid, groups=groups, temp=temp, rho=rho, tables=tables, prt=prt, isv=isv, params=params)


ATOMIC_NPZ = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "atomic_data.npz")


def atomic_data():
    """The reference's atomic data (Verner, Sutherland, data.ion, a subset of
    Data/Atoms lines), from the committed fixture tests/golden/atomic_data.npz."""
    return W.load_atomic_data(ATOMIC_NPZ)


def reference_opacity_case(oracle, ncell=64, ng=200, nline=20000, seed=11, t_days=10.0, lines="reference"):
    """opacity_case on the reference's atomic data: real Verner and Sutherland
    tables, Saha populations (ions_solve_eos + eos_update, via the oracle) from
    the real data.ion levels for every stage below the bare ion, and either the
    real line subset (lines="reference", nline ignored) or nline synthetic lines."""
    import dataclasses
    A = atomic_data()
    case = W.opacity_case(ncell=ncell, ng=ng, nline=nline if lines != "reference" else 1, seed=seed,
                          t_days=t_days, tables=A.tables)
    if lines == "reference":
        case = dataclasses.replace(case, lines=A.lines)
    g = case.gas
    ion = A.ion
    q = oracle.partition(ion, float(g.temp[0]))
    nel, oc, ginv, it = oracle.saha_eos(ion, q, g.temp, g.natom, case.grid.vol, g.natomfr, np.ones(ncell),
                                        acc=1e-12, noc=ion.nstage - 1)
    gas = dataclasses.replace(g, nelec=nel, ion_ni=np.ascontiguousarray(ion.ni, dtype=np.int32), oc=oc, ginv=ginv)
    return dataclasses.replace(case, gas=gas)
