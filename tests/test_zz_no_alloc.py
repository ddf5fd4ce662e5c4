"""slg_particle_advance_static: the particle loop for callers that may not
allocate device memory (a host code whose memory pool owns every device buffer,
or a run where another component owns the allocator).  It keeps its tables and
counters in a fixed __device__ array instead of allocating.  Checked here
through the C ABI against the context-based slg_dev_particle_advance, on two
calls in a row (the shared array must be cleared between calls), with the
transport tolerances of tests/test_gpu_transport.py.
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

import cases
from superlite_b200 import capi
from superlite_b200.capi import ptr

pytestmark = pytest.mark.gpu


def _dev(t, torch, dtype=None):
    return torch.as_tensor(np.ascontiguousarray(t), dtype=dtype, device="cuda")


def _run_existing(hot, c, tables, prt_t, isv_t, seed, torch):
    nx, ng = c["grid"].nx, c["groups"].ng
    tally = torch.zeros(nx, dtype=torch.float64, device="cuda")
    jrad = torch.zeros((nx, ng), dtype=torch.float64, device="cuda")
    eamp = torch.zeros(nx, dtype=torch.float64, device="cuda")
    mswap = torch.zeros(nx, dtype=torch.int32, device="cuda") if c["params"].dogrdtally else None
    out = hot.particle_advance_dev(tables, prt_t, isv_t, tally, jrad, eamp, c["params"], seed=seed,
                                   methodswap=mswap)
    hot.sync()
    return out, tally, jrad, mswap


def _run_static(lib, c, tables, prt_t, isv_t, seed, torch, grid_arrays):
    nx, ng = c["grid"].nx, c["groups"].ng
    g = capi.SlgGridDev(nx, ng, *[ptr(grid_arrays[k]) for k in ("xarr", "vxarr", "divv", "wl", "wlinv")])
    p = c["params"]
    tin = capi.SlgTransportIn(ptr(tables["tempinv"]), ptr(tables["sig"]), ptr(tables["capgrey"]),
                              ptr(tables["emitprob"]), ptr(tables["opaclump"]), ptr(tables["cap"]), p.tauddmc,
                              p.taulump, int(p.puretran), int(p.noampfact), int(p.errorfatal), int(p.thm_aniso),
                              int(p.dogrdtally), 0, int(p.max_steps))
    tally = torch.full((nx,), 7.0, dtype=torch.float64, device="cuda")   # must be overwritten
    jrad = torch.full((nx, ng), 7.0, dtype=torch.float64, device="cuda")
    eamp = torch.full((nx,), 7.0, dtype=torch.float64, device="cuda")
    mswap = torch.full((nx,), 7, dtype=torch.int32, device="cuda") if p.dogrdtally else None
    out = capi.SlgTransportOut(ptr(tally), ptr(jrad), ptr(eamp), ptr(mswap), 0.0, 0.0, 0.0)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.slg_particle_advance_static(C.byref(g), C.byref(tin), ptr(prt_t), ptr(isv_t), int(prt_t.shape[0]),
                                         seed, C.byref(out), C.c_void_p(stream))
    assert rc == 0, rc
    return out, tally, jrad, mswap


@pytest.mark.parametrize("dogrdtally", [False, True])
def test_static_scratch_entry_point_matches_context_entry_point(hot, oracle, dogrdtally):
    import torch
    lib = capi.load()
    c = cases.transport_case(oracle, t_days=6.0, npart=6000, kind="mono")
    c["params"] = dataclasses.replace(c["params"], dogrdtally=dogrdtally)
    hot.set_groups(c["groups"].wl)
    hot.set_grid(c["grid"].xarr, c["grid"].vxarr, c["grid"].vol, c["grid"].divv)
    t = c["tables"]
    tables = dict(tempinv=_dev(t["tempinv"], torch), sig=_dev(t["sig"], torch), capgrey=_dev(t["capgrey"], torch),
                  emitprob=_dev(t["emitprob"], torch), opaclump=_dev(t["opaclump"], torch),
                  cap=_dev(t["cap"], torch, torch.float32))
    grid_arrays = dict(xarr=_dev(c["grid"].xarr, torch), vxarr=_dev(c["grid"].vxarr, torch),
                       divv=_dev(c["grid"].divv, torch), wl=_dev(c["groups"].wl, torch),
                       wlinv=_dev(c["groups"].wlinv, torch))
    prt0 = torch.as_tensor(c["prt"].view(np.float64).reshape(-1, 8)).cuda()
    isv0 = torch.as_tensor(c["isv"]).cuda()
    for seed in (11, 12):  # two calls in a row on the shared array
        pa, va = prt0.clone(), isv0.clone()
        oa, ta, ja, ma = _run_existing(hot, c, tables, pa, va, seed, torch)
        pb, vb = prt0.clone(), isv0.clone()
        ob, tb, jb, mb = _run_static(lib, c, tables, pb, vb, seed, torch, grid_arrays)
        torch.cuda.synchronize()
        assert oa.nstepimc + oa.nstepddmc > 6000
        for k in ("npckt", "nflux", "nstepimc", "nstepddmc", "nmethodswap", "nstepmax", "nposwarn", "ierr"):
            assert getattr(ob, k) == getattr(oa, k), k
        assert list(ob.ndist) == list(oa.ndist)
        assert np.array_equal(vb.cpu().numpy(), va.cpu().numpy())
        live = (va == 0).cpu().numpy()
        np.testing.assert_allclose(pb.cpu().numpy()[live], pa.cpu().numpy()[live], rtol=1e-10, atol=0)
        for k in ("tot_evelo", "tot_eout", "tot_sflux"):
            assert getattr(ob, k) == pytest.approx(getattr(oa, k), rel=1e-9), k
        np.testing.assert_allclose(tb.cpu().numpy(), ta.cpu().numpy(), rtol=1e-9, atol=1e-300)
        np.testing.assert_allclose(jb.cpu().numpy(), ja.cpu().numpy(), rtol=1e-9, atol=1e-300)
        if dogrdtally:  # grd_methodswap per cell, cleared by the call (it started at 7)
            assert np.array_equal(mb.cpu().numpy(), ma.cpu().numpy())
            assert int(ma.sum()) == oa.nmethodswap > 0


def test_static_scratch_rejects_large_grids():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = capi.load()
    big = capi.SlgGridDev(400, 2000, 1, 1, 1, 1, 1)  # 800000 cell-groups > SLG_STATIC_MAX_CELLGROUPS
    tin = capi.SlgTransportIn(1, 1, 1, 1, 1, 1, 5.0, 10.0, 0, 1, 1, 0, 0, 0, 0)
    out = capi.SlgTransportOut(1, 1, 1, None, 0.0, 0.0, 0.0)
    rc = lib.slg_particle_advance_static(C.byref(big), C.byref(tin), 1, 1, 10, 1, C.byref(out), None)
    assert rc == -7  # SLG_ERR_TOO_LARGE, before any device work
    # within the cell-group budget but beyond SLG_MAX_GROUPS (group lists are int16)
    wide = capi.SlgGridDev(2, 40000, 1, 1, 1, 1, 1)
    rc = lib.slg_particle_advance_static(C.byref(wide), C.byref(tin), 1, 1, 10, 1, C.byref(out), None)
    assert rc == -7
