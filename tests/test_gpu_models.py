"""Several models in one context (slg_set_models) against one context per model.

Each model of a batch runs the same per-cell and per-particle arithmetic as
its own single-model run: model m draws its random numbers under the key
seed + m * SLG_MODEL_SEED_STRIDE with slots counted from the model's first
slot.  So opacities, leakage coefficients, source particles and the particle
states after the transport (FP64 or mixed precision) are bit-identical;
tallies and luminosities are sums formed with atomics in a different order
(rtol 1e-12).
"""
import numpy as np
import pytest

from superlite_b200 import HotPath, PACKET_DTYPE
from superlite_b200 import workloads as W

pytestmark = pytest.mark.gpu

STRIDE = 0x9E3779B97F4A7C15
MASK = (1 << 64) - 1
L_BOL = 1e42


def _tables(hot, temp, natom, nelec, vol, mass, natomfr, oc, ginv):
    op = hot.physical_opacity(temp, natom, nelec, vol, mass, natomfr, oc, ginv)
    grey, _ = hot.opacity_means(temp, op["sig"], op["cap"])
    tinv = 1.0 / temp
    ol = hot.leakage_opacity(tinv, op["sig"], op["cap"])
    ep = hot.emission_probability(tinv, op["cap"], grey)
    return dict(tempinv=tinv, sig=op["sig"], capgrey=grey, emitprob=ep, opaclump=ol, cap=op["cap"])


def _run_batch(b, seed_src, seed_tr, params, precision=1):
    hot = HotPath(0)
    hot.set_groups(b.groups.wl)
    hot.set_models(b.nx, b.npart, b.xarr, b.vxarr, b.vol, b.divv)
    c0 = b.models[0]
    hot.set_atomic_data(c0.gas.ion_ni, c0.gas.oc.shape[1], c0.lines, c0.bf_ph1, c0.bf_ph2, c0.ff_gff)
    g = b.gas
    tab = _tables(hot, g.temp, g.natom, g.nelec, b.vol, g.mass, g.natomfr, g.oc, g.ginv)
    emit, _ = hot.sourceenergy(g.temp, L_BOL)
    nvol, nnew = hot.models_sourcenumbers(emit, b.npart)
    n = int(b.npart.sum())
    prt = np.zeros(n, dtype=PACKET_DTYPE)
    isv = np.ones(n, dtype=np.int32)
    hot.interior_source(g.temp, emit, nvol, prt, isv, seed=seed_src)
    src = prt.copy()
    r = hot.particle_advance(tab, prt, isv, params, seed=seed_tr, precision=precision)
    lum, dev, num = hot.fluxtally(prt, isv, b.groups.wl)
    hot.close()
    return dict(tab=tab, emit=emit, nvol=nvol, nnew=nnew, src=src, prt=prt, isv=isv, r=r, lum=lum, dev=dev, num=num)


def _run_one(c, npart, seed_src, seed_tr, params, precision=1):
    hot = HotPath(0)
    hot.set_groups(c.groups.wl)
    hot.set_grid(c.grid.xarr, c.grid.vxarr, c.grid.vol, c.grid.divv)
    hot.set_atomic_data(c.gas.ion_ni, c.gas.oc.shape[1], c.lines, c.bf_ph1, c.bf_ph2, c.ff_gff)
    g = c.gas
    tab = _tables(hot, g.temp, g.natom, g.nelec, c.grid.vol, g.mass, g.natomfr, g.oc, g.ginv)
    emit, _ = hot.sourceenergy(g.temp, L_BOL)
    nvol, nnew = hot.sourcenumbers(emit, npart)
    prt = np.zeros(npart, dtype=PACKET_DTYPE)
    isv = np.ones(npart, dtype=np.int32)
    hot.interior_source(g.temp, emit, nvol, prt, isv, seed=seed_src)
    src = prt.copy()
    r = hot.particle_advance(tab, prt, isv, params, seed=seed_tr, precision=precision)
    lum, dev, num = hot.fluxtally(prt, isv, c.groups.wl)
    hot.close()
    return dict(tab=tab, emit=emit, nvol=nvol, nnew=nnew, src=src, prt=prt, isv=isv, r=r, lum=lum, dev=dev, num=num)


@pytest.mark.parametrize("precision", [1, 0])
@pytest.mark.parametrize("t_days", [(4.0, 8.0), (15.0, 30.0)])
def test_models_match_single_model_runs(t_days, precision):
    b = W.model_batch(nmodel=3, seed=9, ng=100, nline=20000, nx=[20, 35, 50], npart=[3000, 5000, 2000],
                      t_range_days=t_days)
    params = W.TransportParams()
    s_src, s_tr = 77, 1234
    B = _run_batch(b, s_src, s_tr, params, precision)
    assert B["r"]["ierr"] == 0
    steps = 0
    for m, c in enumerate(b.models):
        co = int(b.nx[:m].sum())
        cs = slice(co, co + int(b.nx[m]))
        po = int(b.npart[:m].sum())
        ps = slice(po, po + int(b.npart[m]))
        S = _run_one(c, int(b.npart[m]), (s_src + m * STRIDE) & MASK, (s_tr + m * STRIDE) & MASK, params,
                     precision)
        assert S["r"]["ierr"] == 0
        for k in ("sig", "capgrey", "opaclump", "emitprob", "cap"):
            np.testing.assert_array_equal(B["tab"][k][cs], S["tab"][k], err_msg=k)
        np.testing.assert_array_equal(B["emit"][cs], S["emit"])
        np.testing.assert_array_equal(B["nvol"][cs], S["nvol"])
        np.testing.assert_array_equal(B["src"][ps].view(np.float64), S["src"].view(np.float64))
        np.testing.assert_array_equal(B["prt"][ps].view(np.float64), S["prt"].view(np.float64))
        np.testing.assert_array_equal(B["isv"][ps], S["isv"])
        np.testing.assert_allclose(B["lum"][m], S["lum"], rtol=1e-12, atol=0)
        np.testing.assert_allclose(B["dev"][m], S["dev"], rtol=1e-12, atol=0)
        np.testing.assert_array_equal(B["num"][m], S["num"])
        np.testing.assert_allclose(B["r"]["tally"][cs], S["r"]["tally"], rtol=1e-12, atol=0)
        steps += S["r"]["nstepimc"] + S["r"]["nstepddmc"]
    assert B["r"]["nstepimc"] + B["r"]["nstepddmc"] == steps


def test_models_source_stays_in_model_slots():
    """A model with fewer vacancies than new particles is an error; other
    models' free slots are never borrowed."""
    b = W.model_batch(nmodel=2, seed=3, ng=50, nline=5000, nx=[10, 12], npart=[400, 400])
    hot = HotPath(0)
    hot.set_groups(b.groups.wl)
    hot.set_models(b.nx, b.npart, b.xarr, b.vxarr, b.vol, b.divv)
    emit, _ = hot.sourceenergy(b.gas.temp, L_BOL)
    nvol, nnew = hot.models_sourcenumbers(emit, [400, 400])
    prt = np.zeros(800, dtype=PACKET_DTYPE)
    isv = np.ones(800, dtype=np.int32)
    isv[:200] = 0  # model 0 has only 200 vacancies
    from superlite_b200.capi import SlgError
    with pytest.raises(SlgError):
        hot.interior_source(b.gas.temp, emit, nvol, prt, isv, seed=1)
    hot.close()


@pytest.mark.parametrize("precision", [1, 0])
def test_models_edge_cases(precision):
    """Ragged batches: two- and three-shell models beside a 40-shell one, and a
    call whose slots are all vacant (nothing to transport, zero counters)."""
    params = W.TransportParams()
    b = W.analytic_batch(nmodel=3, seed=11, nx=[2, 40, 3], npart=[1000, 3000, 500], t_range_days=(6.0, 12.0))
    hot = HotPath(0)
    hot.set_groups(b.groups.wl)
    hot.set_models(b.nx, b.npart, b.xarr, b.vxarr, b.vol, b.divv)
    sig, cap = hot.analytic_opacity(b.temp, b.rho, kind=1)
    grey, _ = hot.opacity_means(b.temp, sig, cap)
    tinv = 1.0 / b.temp
    ol = hot.leakage_opacity(tinv, sig, cap)
    ep = hot.emission_probability(tinv, cap, grey)
    tab = dict(tempinv=tinv, sig=sig, capgrey=grey, emitprob=ep, opaclump=ol, cap=cap)
    n = int(b.npart.sum())
    prt = np.zeros(n, dtype=PACKET_DTYPE)
    isv = np.ones(n, dtype=np.int32)
    # all slots vacant: the loop has nothing to do
    r0 = hot.particle_advance(tab, prt, isv, params, seed=1, precision=precision)
    assert r0["ierr"] == 0 and r0["npckt"] == 0 and r0["nstepimc"] + r0["nstepddmc"] == 0
    # sources in every model, then one step over all three
    emit, _ = hot.sourceenergy(b.temp, L_BOL)
    nvol, nnew = hot.models_sourcenumbers(emit, b.npart)
    assert nnew <= n
    hot.interior_source(b.temp, emit, nvol, prt, isv, seed=2)
    assert int((isv == 0).sum()) == nnew
    r = hot.particle_advance(tab, prt, isv, params, seed=3, precision=precision)
    assert r["ierr"] == 0 and r["npckt"] == nnew
    lum, dev, num = hot.fluxtally(prt, isv, b.groups.wl)
    lum = np.asarray(lum).reshape(3, -1)
    assert np.all(lum.sum(axis=1) > 0.0)
    assert np.all(isv == 1)               # every particle escaped or was absorbed and freed
    hot.close()
