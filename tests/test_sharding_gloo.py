"""Two-rank (gloo, CPU) check of the particle sharding used by bench.py --gpus N:
each rank transports its own slice of the particles (oracle, shared Philox
stream keyed by the global particle index) and the tallies are summed with an
all-reduce; the result must equal one process transporting all particles."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle"), os.path.join(root, "tests")):
        sys.path.insert(0, p)
    import torch
    import torch.distributed as dist
    import pyoracle as po
    import cases
    from superlite_b200 import sharding
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = cases.transport_case(po, t_days=8.0, npart=3001)
        lo, hi = sharding.shard_range(3001, rank, world)
        prt, isv = c["prt"].copy(), c["isv"].copy()
        isv[:lo] = 1
        isv[hi:] = 1  # other ranks' slots are vacant here
        tt = po.TransportTables(c["grid"], c["groups"], **c["tables"], params=c["params"])
        r = po.particle_advance(tt, prt, isv, rngmode=1, seed=9, nthreads=2)
        lum, dev, num = po.fluxtally(prt, isv, c["groups"].wl)
        ts = [torch.tensor(r["tally"]), torch.tensor(r["jrad"]), torch.tensor(lum), torch.tensor(dev),
              torch.tensor(num.astype(np.float64))]
        sharding.reduce_tallies(ts)
        cnt = sharding.reduce_counters(r, "cpu")
        if rank == 0:
            q.put(([t.numpy() for t in ts], cnt))
    finally:
        dist.destroy_process_group()


def test_two_rank_tallies_equal_single_process(oracle):
    import cases
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, cnt = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    c = cases.transport_case(oracle, t_days=8.0, npart=3001)
    prt, isv = c["prt"].copy(), c["isv"].copy()
    tt = oracle.TransportTables(c["grid"], c["groups"], **c["tables"], params=c["params"])
    r = oracle.particle_advance(tt, prt, isv, rngmode=1, seed=9, nthreads=2)
    lum, dev, num = oracle.fluxtally(prt, isv, c["groups"].wl)
    np.testing.assert_allclose(got[0], r["tally"], rtol=1e-11, atol=1e-300)
    np.testing.assert_allclose(got[1], r["jrad"], rtol=1e-11, atol=1e-300)
    np.testing.assert_allclose(got[2], lum, rtol=1e-12, atol=0)
    np.testing.assert_allclose(got[3], dev, rtol=1e-12, atol=0)
    assert np.array_equal(got[4], num)
    for k in ("npckt", "nflux", "nstepimc", "nstepddmc", "nstepmax"):
        assert cnt[k] == r[k], k


def test_shard_ranges_cover_all():
    from superlite_b200 import sharding
    for n, w in [(10, 3), (7, 8), (1000003, 8)]:
        rs = [sharding.shard_range(n, k, w) for k in range(w)]
        assert rs[0][0] == 0 and rs[-1][1] == n
        assert all(rs[k][1] == rs[k + 1][0] for k in range(w - 1))
        assert max(b - a for a, b in rs) - min(b - a for a, b in rs) <= 1


def _opacity_worker(rank, world, port, q):
    import dataclasses
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle"), os.path.join(root, "tests")):
        sys.path.insert(0, p)
    import torch
    import torch.distributed as dist
    import pyoracle as po
    from superlite_b200 import sharding, workloads as W
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        case = W.opacity_case(ncell=37, ng=60, nline=3000, seed=13)
        lo, hi = sharding.shard_cells(case.grid.nx, rank, world)
        g, gr = case.gas, case.grid
        sub_grid = dataclasses.replace(gr, nx=hi - lo, xarr=gr.xarr[lo:hi + 1], vxarr=gr.vxarr[lo:hi + 1],
                                       vol=gr.vol[lo:hi], divv=gr.divv[lo:hi])
        sub_gas = dataclasses.replace(g, temp=g.temp[lo:hi], mass=g.mass[lo:hi], rho=g.rho[lo:hi],
                                      natom=g.natom[lo:hi], nelec=g.nelec[lo:hi], natomfr=g.natomfr[lo:hi],
                                      massfr=g.massfr[lo:hi], oc=g.oc[:, :, lo:hi], ginv=g.ginv[:, :, lo:hi])
        r = po.physical_opacity(dataclasses.replace(case, grid=sub_grid, gas=sub_gas))
        got = [sharding.gather_cells(torch.tensor(r[k]), case.grid.nx) for k in ("cap", "sig", "cap64")]
        if rank == 0:
            q.put([t.numpy() for t in got])
    finally:
        dist.destroy_process_group()


def test_two_rank_cell_sharded_opacity_equals_single_process(oracle):
    """Opacity sharded by shells (each rank builds its shells, then one
    all-gather) equals the single-process build bit for bit: the opacity of a
    shell depends on that shell alone."""
    from superlite_b200 import workloads as W
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_opacity_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    ref = oracle.physical_opacity(W.opacity_case(ncell=37, ng=60, nline=3000, seed=13))
    assert np.array_equal(got[0], ref["cap"])
    assert np.array_equal(got[1], ref["sig"])
    assert np.array_equal(got[2], ref["cap64"])
