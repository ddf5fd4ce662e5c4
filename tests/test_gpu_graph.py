"""CUDA-graph capture of whole timesteps (slg_graph_begin/end/launch).

Replay 0 of a captured sequence equals the same calls made directly (same
kernels, same random numbers); later replays draw from fresh Philox counters.
Transport counters of replays accumulate in slg_transport_totals.
"""
import numpy as np
import pytest
import torch

from superlite_b200 import HotPath
from superlite_b200 import workloads as W
from superlite_b200.timestep import DeviceTimestep

pytestmark = pytest.mark.gpu

L_BOL = 1e42


def _setup(precision, npart=20000):
    case = W.opacity_case(ncell=48, ng=120, nline=20000, seed=5, t_days=12.0)
    hot = HotPath(0)
    ts = DeviceTimestep(hot, case, W.TransportParams(), npart=npart, precision=precision)
    emit, _ = hot.sourceenergy(case.gas.temp, L_BOL)
    nvol, _ = hot.sourcenumbers(emit, npart)
    ts.isv.fill_(1)
    return hot, ts, emit, nvol


def _step(hot, ts, emit, nvol, k):
    hot.interior_source(ts.gas["temp"], emit, nvol, ts.prt, ts.isv, seed=100 + k)
    ts.opacity()
    ts.coefficients()
    ts.transport(200 + k)
    ts.fluxtally()


KEYS = ("npckt", "nflux", "nstepimc", "nstepddmc", "nstepmax", "nmethodswap")


@pytest.mark.parametrize("precision", [0, 1])
def test_graph_replay_equals_direct_calls(precision):
    hot, ts, emit, nvol = _setup(precision)
    direct = []
    for k in range(2):  # uncaptured pass: every buffer and upload exists afterwards
        _step(hot, ts, emit, nvol, k)
        c = ts.sync()
        direct.append((ts.prt.clone(), ts.lum.clone(), ts.tally.clone(), {q: c[q] for q in KEYS}))
    hot.transport_totals(reset=True)
    hot.graph_begin()
    for k in range(2):
        _step(hot, ts, emit, nvol, k)
    hot.graph_end()
    hot.graph_launch(1)
    hot.sync()
    prt, lum, tally, cnt = direct[-1]
    assert torch.equal(ts.prt, prt)
    torch.testing.assert_close(ts.lum, lum, rtol=1e-12, atol=0)
    torch.testing.assert_close(ts.tally, tally, rtol=1e-12, atol=0)
    tot = hot.transport_totals(reset=True)
    assert tot["ierr"] == 0
    for q in ("npckt", "nflux", "nstepimc", "nstepddmc", "nmethodswap"):
        assert tot[q] == direct[0][3][q] + direct[1][3][q], q
    assert tot["nstepmax"] == max(direct[0][3]["nstepmax"], direct[1][3]["nstepmax"])
    # replay 1: fresh random numbers, same physics
    hot.graph_launch(1)
    hot.sync()
    assert not torch.equal(ts.prt, prt)
    tot2 = hot.transport_totals()
    assert tot2["npckt"] == tot["npckt"]
    s1 = (tot["nstepimc"] + tot["nstepddmc"]) / tot["npckt"]
    s2 = (tot2["nstepimc"] + tot2["nstepddmc"]) / tot2["npckt"]
    assert s2 == pytest.approx(s1, rel=0.1)
    hot.close()


def test_graph_capture_rejects_changed_upload():
    """A changed source set-up needs a host upload, which a capture cannot hold."""
    hot, ts, emit, nvol = _setup(1, npart=5000)
    _step(hot, ts, emit, nvol, 0)
    ts.sync()
    hot.graph_begin()
    from superlite_b200.capi import SlgError
    with pytest.raises(SlgError):
        hot.interior_source(ts.gas["temp"], emit * 1.5, nvol, ts.prt, ts.isv, seed=3)
    with pytest.raises(SlgError):
        hot.graph_end()
    # the context stays usable
    _step(hot, ts, emit, nvol, 1)
    assert ts.sync()["ierr"] == 0
    hot.close()


def test_autotuner_leaves_particles_and_picks_a_variant():
    """slg_autotune_transport (HotPath.autotune_transport) times every variant on
    a copy: the caller's particles and vacancy flags are unchanged."""
    from superlite_b200.timestep import BatchTimestep
    b = W.analytic_batch(nmodel=2, seed=4, nx=[20, 30], npart=[2000, 3000], t_range_days=(5.0, 10.0))
    hot = HotPath(0)
    params = W.TransportParams()
    ts = BatchTimestep(hot, b, params, precision=1)
    ts.prepare(3)
    ts.sync()
    before_p, before_v = ts.prt.clone(), ts.isv.clone()
    tables = dict(tempinv=ts.tempinv, sig=ts.sig, capgrey=ts.capgrey, emitprob=ts.emitprob, opaclump=ts.opaclump,
                  cap=ts.cap)
    v, ms = hot.autotune_transport(tables, ts.prt, ts.isv, params, precision=1, seed=3, nsample=4000)
    hot.sync()
    assert 0 <= v < 4 and all(m > 0.0 for m in ms)
    assert torch.equal(ts.prt, before_p) and torch.equal(ts.isv, before_v)
    hot.close()
