"""Seeded parity cases shared by the GPU tests (small enough for the oracle)."""
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
