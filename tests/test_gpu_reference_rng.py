"""The GPU particle loop (Philox streams) against the oracle run with the
reference's own random-number generator (mzran, randommod.f:73-92, one stream
per OpenMP thread as particle_advance.f90:87-140 draws them), at matched
particle counts on the CPU-runnable workload's physics (64 shells, 100 groups,
analytic grey opacity).

The two runs share the source particles and differ only in the random numbers,
so they agree in distribution, not event by event.  K = 10 independent runs of
each: group luminosities in 10 wavelength bins, summed over the runs, within 3
sigma of the Monte Carlo noise estimated from lumdev (fluxtally.f:47-49); the
deposited energy (grd_tally) in 4 shell bins, the escaped energy and the steps
per particle within 3 sigma of the K-run batch variance (Welch t; 18 degrees
of freedom).  False-alarm rate of the 17 comparisons of one snapshot under the
null: 10 x 0.27 % (normal) + 7 x 0.77 % (t with 18 dof), about 8 %; the seeds
are fixed, so each run of the test is deterministic.
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

K = 10


def _binned(lum, nbin=10):
    edges = np.linspace(0, len(lum), nbin + 1).astype(int)
    return np.array([lum[a:b].sum() for a, b in zip(edges[:-1], edges[1:])])


def _welch(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    se = np.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
    return (a.mean() - b.mean()) / se if se > 0 else 0.0


@pytest.mark.parametrize("t_days", [2.0, 10.0])
def test_fp64_loop_matches_oracle_with_reference_rng(hot, oracle, t_days):
    c = cases.transport_case(oracle, t_days=t_days, npart=20000)
    hot.set_groups(c["groups"].wl)
    hot.set_grid(c["grid"].xarr, c["grid"].vxarr, c["grid"].vol, c["grid"].divv)
    tt = oracle.TransportTables(c["grid"], c["groups"], **c["tables"], params=c["params"])
    nthreads = 8
    runs = {"mzran": [], "gpu": []}
    for k in range(K):
        po, vo = c["prt"].copy(), c["isv"].copy()
        st = oracle.rnd_init(nthreads, 1 + k)  # disjoint mzran seeds per run and thread
        r = oracle.particle_advance(tt, po, vo, rngmode=0, nthreads=nthreads, rnd_states=st)
        lum, dev, num = oracle.fluxtally(po, vo, c["groups"].wl)
        runs["mzran"].append((r, lum, dev))
        pg, vg = c["prt"].copy(), c["isv"].copy()
        r = hot.particle_advance(c["tables"], pg, vg, c["params"], seed=500 + k)
        lum, dev, num = hot.fluxtally(pg, vg, c["groups"].wl)
        runs["gpu"].append((r, lum, dev))
    for name in runs:
        for r, _, _ in runs[name]:
            assert r["ierr"] == 0 and r["npckt"] == 20000
    # binned group luminosities with the fluxtally noise
    la = sum(_binned(l) for _, l, _ in runs["mzran"])
    va = sum(_binned(d) for _, _, d in runs["mzran"])
    lb = sum(_binned(l) for _, l, _ in runs["gpu"])
    vb = sum(_binned(d) for _, _, d in runs["gpu"])
    ok = va + vb > 0
    z = (la - lb)[ok] / np.sqrt((va + vb)[ok])
    assert np.all(np.abs(z) < 3.0), z
    # deposition per shell bin, escaped energy and steps per particle with the K-run variance
    nx = c["grid"].nx
    edges = np.linspace(0, nx, 5).astype(int)
    for a, b in zip(edges[:-1], edges[1:]):
        d0 = [r["tally"][a:b].sum() for r, _, _ in runs["mzran"]]
        d1 = [r["tally"][a:b].sum() for r, _, _ in runs["gpu"]]
        assert abs(_welch(d0, d1)) < 3.0, (a, b, d0, d1)
    esc = {n: [l.sum() for _, l, _ in runs[n]] for n in runs}
    assert abs(_welch(esc["mzran"], esc["gpu"])) < 3.0, esc
    steps = {n: [(r["nstepimc"] + r["nstepddmc"]) / r["npckt"] for r, _, _ in runs[n]] for n in runs}
    assert abs(_welch(steps["mzran"], steps["gpu"])) < 3.0, steps
