"""The CUDA path against the committed golden fixtures (tests/golden/): the
oracle's outputs for small seeded cases, so these checks run no oracle
opacity build or particle loop at test time."""
import os

import numpy as np
import pytest

import cases
from superlite_b200 import HotPath
from superlite_b200 import workloads as W

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "oracle_small.npz")


def test_opacity_matches_golden():
    g = np.load(GOLD)
    oc = W.opacity_case(ncell=8, ng=24, nline=400, seed=31, t_days=9.0)
    hot = HotPath(0)
    hot.set_groups(oc.groups.wl)
    hot.set_grid(oc.grid.xarr, oc.grid.vxarr, oc.grid.vol, oc.grid.divv)
    gas = oc.gas
    hot.set_atomic_data(gas.ion_ni, gas.oc.shape[1], oc.lines, oc.bf_ph1, oc.bf_ph2, oc.ff_gff)
    r = hot.physical_opacity(gas.temp, gas.natom, gas.nelec, oc.grid.vol, gas.mass, gas.natomfr, gas.oc, gas.ginv,
                             want_cap64=True)
    np.testing.assert_allclose(r["cap64"], g["opac_cap64"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(r["sig"], g["opac_sig"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(r["cap"], g["opac_cap"], rtol=2.4e-7, atol=0)  # 1 float ulp
    hot.close()


def test_event_sequences_match_golden(oracle):
    g = np.load(GOLD)
    c = cases.transport_case(oracle, t_days=6.0, nx=16, ng=20, npart=300, seed=5)
    hot = HotPath(0)
    hot.set_groups(c["groups"].wl)
    hot.set_grid(c["grid"].xarr, c["grid"].vxarr, c["grid"].vol, c["grid"].divv)
    prt, isv = c["prt"].copy(), c["isv"].copy()
    r = hot.particle_advance(c["tables"], prt, isv, c["params"], seed=7, trace=True)
    assert np.array_equal(r["trace_hash"], g["trn_trace_hash"])
    got = np.array([r["npckt"], r["nflux"], r["nstepimc"], r["nstepddmc"], r["nstepmax"]], dtype=np.int64)
    assert np.array_equal(got, g["trn_counts"])
    np.testing.assert_allclose(r["tally"], g["trn_tally"], rtol=1e-9, atol=1e-300)
    hot.close()
