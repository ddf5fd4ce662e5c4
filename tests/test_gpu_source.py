"""GPU source-particle creation (vacancies + interior_source +
source_transformdirection) against the oracle run with the same per-particle
Philox streams, and the host-side sourceenergy / sourcenumbers."""
import numpy as np
import pytest

from superlite_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _case(nx=64, ng=100, t_days=5.0, seed=3):
    grid = W.homologous_grid(nx, t_days * W.PC_DAY)
    groups = W.group_grid(ng)
    temp = np.random.default_rng(seed).uniform(6000.0, 14000.0, nx)
    return grid, groups, temp


def _setup(hot, grid, groups):
    hot.set_groups(groups.wl)
    hot.set_grid(grid.xarr, grid.vxarr, grid.vol, grid.divv)


def test_sourceenergy_and_numbers_match_oracle(hot, oracle):
    grid, groups, temp = _case()
    _setup(hot, grid, groups)
    emit, tot = hot.sourceenergy(temp, 1e42)
    lib = oracle.lib()
    e_ref = np.zeros(grid.nx)
    t_ref = np.zeros(1)
    lib.orc_sourceenergy(grid.nx, grid.xarr.ctypes.data_as(oracle.dp), temp.ctypes.data_as(oracle.dp), 1e42,
                         e_ref.ctypes.data_as(oracle.dp), t_ref.ctypes.data_as(oracle.dp))
    assert np.array_equal(emit, e_ref) and tot == t_ref[0]
    for ns in (64, 1000, 123457):
        nvol, nnew = hot.sourcenumbers(emit, ns)
        nv_ref = np.zeros(grid.nx, dtype=np.int32)
        n_ref = lib.orc_sourcenumbers(grid.nx, emit.ctypes.data_as(oracle.dp), 1.0, ns, ns,
                                      nv_ref.ctypes.data_as(oracle.ip))
        assert nnew == n_ref == ns
        assert np.array_equal(nvol, nv_ref)


@pytest.mark.parametrize("ng,npart,prefill", [(100, 20000, 0), (300, 7000, 3000)])
def test_interior_source_matches_oracle(hot, oracle, ng, npart, prefill):
    grid, groups, temp = _case(ng=ng)
    _setup(hot, grid, groups)
    emit, _ = hot.sourceenergy(temp, 1e42)
    nvol, nnew = hot.sourcenumbers(emit, npart - prefill)
    # some occupied slots to exercise the vacancy list
    isv0 = np.ones(npart, dtype=np.int32)
    occ = np.random.default_rng(1).choice(npart, prefill, replace=False)
    isv0[occ] = 0
    from superlite_b200 import PACKET_DTYPE
    prt = np.zeros(npart, dtype=PACKET_DTYPE)
    prt["x"][occ] = 12345.0
    isv = isv0.copy()
    n = hot.interior_source(temp, emit, nvol, prt, isv, seed=77)
    assert n == nnew
    ref, isv_ref, *_ = oracle.make_source_particles(grid, groups, temp, 1e42, npart - prefill, npart=npart,
                                                    rngmode=1, seed=77, isvacant=isv0)
    assert np.array_equal(isv, isv_ref)
    new = isv0 == 1
    for f in ("x", "y", "z", "mu", "om", "e", "e0", "wl"):
        np.testing.assert_allclose(prt[f][new], ref[f][new], rtol=1e-14, atol=0, err_msg=f)
    assert np.all(prt["x"][occ] == 12345.0)
    # distribution sanity: energies sum to L_bol, positions inside the grid
    assert prt["e"][new].sum() == pytest.approx(1e42, rel=1e-12)
    assert np.all(prt["x"][new] >= grid.xarr[0]) and np.all(prt["x"][new] <= grid.xarr[-1])


def test_interior_source_rejects_too_few_slots(hot):
    from superlite_b200 import PACKET_DTYPE, SlgError
    grid, groups, temp = _case()
    _setup(hot, grid, groups)
    emit, _ = hot.sourceenergy(temp, 1e42)
    nvol, nnew = hot.sourcenumbers(emit, 5000)
    prt = np.zeros(4000, dtype=PACKET_DTYPE)
    with pytest.raises(SlgError):
        hot.interior_source(temp, emit, nvol, prt, np.ones(4000, dtype=np.int32), seed=1)
