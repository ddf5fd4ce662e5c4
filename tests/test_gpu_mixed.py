"""Mixed-precision transport (precision=1) against the FP64 form.

The mixed form draws different random numbers (FP32 stream) and rounds
distances, directions and wavelengths in single precision, so it is compared
statistically: group luminosities (binned) within 3 sigma of Monte Carlo noise,
estimated from lumdev = sum of e^2 per group (fluxtally.f:47-49), and the
escaped energy, the deposited energy and the mean number of steps per
particle against the spread of independent runs.

False-alarm rate: 10 luminosity bins at |z| < 3 (0.27 % each under a normal
null) and 7 Welch statistics at |t| < 4 (18 dof, 0.08 % each): about 3 % per
snapshot; the seeds are fixed, so each run of the test is deterministic.
"""
import numpy as np
import pytest

import cases
from superlite_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _run(hot, c, precision, seed):
    pg, vg = c["prt"].copy(), c["isv"].copy()
    r = hot.particle_advance(c["tables"], pg, vg, c["params"], seed=seed, precision=precision)
    lum, dev, num = hot.fluxtally(pg, vg, c["groups"].wl)
    return r, lum, dev, num


def _binned_z(lum_a, dev_a, lum_b, dev_b, nbin=10):
    edges = np.linspace(0, len(lum_a), nbin + 1).astype(int)
    z = []
    for a, b in zip(edges[:-1], edges[1:]):
        la, lb = lum_a[a:b].sum(), lum_b[a:b].sum()
        va, vb = dev_a[a:b].sum(), dev_b[a:b].sum()
        if va + vb > 0:
            z.append((la - lb) / np.sqrt(va + vb))
    return np.array(z)


def _welch(a, b):
    """t statistic of the difference of two means from K independent runs each."""
    a, b = np.asarray(a, float), np.asarray(b, float)
    se = np.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
    return (a.mean() - b.mean()) / se if se > 0 else 0.0


@pytest.mark.parametrize("t_days,kind", [(1.5, "grey"), (5.0, "grey"), (6.0, "mono"), (20.0, "grey+sig")])
def test_mixed_matches_fp64_statistically(hot, oracle, t_days, kind):
    """K independent seeds per form.  Steps per particle and the deposited energy
    have heavy-tailed per-particle distributions (a few per cent spread between
    seeds at 2e4 particles), so they are compared with the K-run batch variance
    (Welch t, |t| < 4 at 2K-2 = 18 degrees of freedom); luminosities use the
    fluxtally variance estimate lumdev."""
    c = cases.transport_case(oracle, t_days=t_days, npart=20000, kind=kind)
    hot.set_groups(c["groups"].wl)
    hot.set_grid(c["grid"].xarr, c["grid"].vxarr, c["grid"].vol, c["grid"].divv)
    K = 10
    runs = {0: [], 1: []}
    for prec in (0, 1):
        for k in range(K):
            r, lum, dev, num = _run(hot, c, prec, 100 * prec + k + 1)
            assert r["ierr"] == 0 and r["npckt"] == c["isv"].size - int(c["isv"].sum())
            runs[prec].append((r, lum, dev))
    steps = {p: [(r["nstepimc"] + r["nstepddmc"]) / r["npckt"] for r, _, _ in runs[p]] for p in runs}
    dep = {p: [r["tally"].sum() for r, _, _ in runs[p]] for p in runs}
    esc = {p: [lum.sum() for _, lum, _ in runs[p]] for p in runs}
    assert abs(_welch(steps[0], steps[1])) < 4.0, (steps[0], steps[1])
    assert abs(_welch(dep[0], dep[1])) < 4.0, (dep[0], dep[1])
    assert abs(_welch(esc[0], esc[1])) < 4.0, (esc[0], esc[1])
    # deposition per shell, in 4 contiguous shell bins (each with enough events
    # that the K-run means are near normal: the per-particle deposition is
    # heavy-tailed in the optically thick cases)
    nx = c["grid"].nx
    edges = np.linspace(0, nx, 5).astype(int)
    for a, b in zip(edges[:-1], edges[1:]):
        d0 = [r["tally"][a:b].sum() for r, _, _ in runs[0]]
        d1 = [r["tally"][a:b].sum() for r, _, _ in runs[1]]
        if max(d0 + d1) > 0:
            assert abs(_welch(d0, d1)) < 4.0, (a, b, d0, d1)
    # group luminosities, summed over the K runs, binned, with lumdev noise
    lum64 = sum(l for _, l, _ in runs[0]); dev64 = sum(d for _, _, d in runs[0])
    lum32 = sum(l for _, l, _ in runs[1]); dev32 = sum(d for _, _, d in runs[1])
    z = _binned_z(lum64, dev64, lum32, dev32)
    assert np.all(np.abs(z) < 3.0), z


def test_mixed_pure_ddmc_full_timestep_physics(hot):
    """The full-timestep case's physics (256 shells x 2000 groups, every shell
    optically thick): the DDMC random walk."""
    from superlite_b200 import PACKET_DTYPE
    case = W.opacity_case(ncell=256, ng=2000, nline=500_000, seed=2, t_days=10.0)
    hot.set_groups(case.groups.wl)
    hot.set_grid(case.grid.xarr, case.grid.vxarr, case.grid.vol, case.grid.divv)
    hot.set_atomic_data(case.gas.ion_ni, case.gas.oc.shape[1], case.lines, case.bf_ph1, case.bf_ph2, case.ff_gff)
    g = case.gas
    op = hot.physical_opacity(g.temp, g.natom, g.nelec, case.grid.vol, g.mass, g.natomfr, g.oc, g.ginv)
    grey, _ = hot.opacity_means(g.temp, op["sig"], op["cap"])
    tinv = 1.0 / g.temp
    ol = hot.leakage_opacity(tinv, op["sig"], op["cap"])
    ep = hot.emission_probability(tinv, op["cap"], grey)
    tables = dict(tempinv=tinv, sig=op["sig"], capgrey=grey, emitprob=ep, opaclump=ol, cap=op["cap"])
    emit, _ = hot.sourceenergy(g.temp, 1e42)
    nvol, n = hot.sourcenumbers(emit, 20000)
    res = []
    for prec, seed in ((0, 5), (1, 6)):
        prt = np.zeros(20000, dtype=PACKET_DTYPE)
        isv = np.ones(20000, dtype=np.int32)
        hot.interior_source(g.temp, emit, nvol, prt, isv, seed=seed)
        r = hot.particle_advance(tables, prt, isv, W.TransportParams(), seed=seed, precision=prec)
        lum, dev, num = hot.fluxtally(prt, isv, case.groups.wl)
        res.append((r, lum, dev))
    (a, la, da), (b, lb, db) = res
    assert a["nstepimc"] == 0 and b["nstepimc"] == 0
    z = _binned_z(la, da, lb, db, nbin=8)
    assert np.all(np.abs(z) < 3.0), z
    sa = a["nstepddmc"] / a["npckt"]
    sb = b["nstepddmc"] / b["npckt"]
    assert sb == pytest.approx(sa, rel=0.05)
