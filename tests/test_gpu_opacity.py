"""GPU parity of the opacity build against the CPU oracle (through the C ABI).

Tolerances: the FP64 opacity before sngl() within 1e-12 relative (the bar the
reference path is held to); the real*4 gas_cap equal to the oracle's except
where the FP64 values straddle a float rounding boundary (at most 1 ulp);
tree-reduced sums (means, leakage) within 1e-11 relative.
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def _setup(hot, case):
    hot.set_groups(case.groups.wl)
    hot.set_grid(case.grid.xarr, case.grid.vxarr, case.grid.vol, case.grid.divv)
    hot.set_atomic_data(case.gas.ion_ni, case.gas.oc.shape[1], case.lines, case.bf_ph1, case.bf_ph2, case.ff_gff)


def _gpu_opacity(hot, case, **kw):
    g = case.gas
    return hot.physical_opacity(g.temp, g.natom, g.nelec, case.grid.vol, g.mass, g.natomfr, g.oc, g.ginv,
                                want_cap64=True, **kw)


def _assert_float_close(a, b, max_ulp=1):
    a = np.asarray(a, dtype=np.float32)
    b = np.asarray(b, dtype=np.float32)
    ia = a.view(np.int32).astype(np.int64)
    ib = b.view(np.int32).astype(np.int64)
    assert np.max(np.abs(ia - ib)) <= max_ulp


def _assert_opacity_parity(got, ref):
    np.testing.assert_allclose(got["sig"], ref["sig"], rtol=1e-15, atol=0)
    pos = ref["cap64"] > 0
    rel = np.abs(got["cap64"][pos] - ref["cap64"][pos]) / ref["cap64"][pos]
    assert rel.max() <= 1e-12, rel.max()
    assert np.array_equal(got["cap64"][~pos], ref["cap64"][~pos])
    _assert_float_close(got["cap"], ref["cap"], 1)
    assert np.mean(got["cap"] == ref["cap"]) > 0.999
    np.testing.assert_allclose(got["emiss"], ref["emiss"], rtol=2e-7, atol=0)
    assert got["sanity"] == ref["flags"]


@pytest.mark.parametrize("flags", [dict(), dict(nobb=True), dict(nobf=True), dict(noff=True),
                                   dict(nothmson=True), dict(ngs=2, opacmixrossel=0.5)])
def test_physical_opacity_matches_oracle(hot, oracle, flags):
    case = cases.opacity_case(ncell=64, ng=200, nline=20000, seed=11)
    _setup(hot, case)
    ref = oracle.physical_opacity(case, **flags)
    got = _gpu_opacity(hot, case, **flags)
    _assert_opacity_parity(got, ref)


@pytest.mark.parametrize("flags", [dict(), dict(nobb=True, noff=True), dict(nobb=True, nobf=True)])
def test_physical_opacity_on_reference_atomic_data(hot, oracle, flags):
    """The reference's own tables: Verner fits (with the nout/einn special
    cases of bfxsmod.f:104-127), Sutherland Gaunt factors (with the clamp of
    physical_opacity.f:238 on the real grid), Saha populations from data.ion
    for all nine bound stages, and 16000 real lines of the ten elements."""
    case = cases.reference_opacity_case(oracle, ncell=64, ng=200, seed=11, lines="reference")
    _setup(hot, case)
    ref = oracle.physical_opacity(case, **flags)
    got = _gpu_opacity(hot, case, **flags)
    assert np.all(ref["cap64"] >= 0) and ref["cap64"].max() > 0
    _assert_opacity_parity(got, ref)


@pytest.mark.parametrize("nrow", [85, 100, 170])
def test_physical_opacity_many_population_rows(hot, oracle, nrow):
    """Lines spread over many ion stages: the forward kernel stages the
    population rows that lines reference in shared memory for up to 160 rows
    (from about 77 rows on, a block needs more than the default 48 KB) and
    reads them from global memory beyond; both against the oracle."""
    import dataclasses
    case = cases.reference_opacity_case(oracle, ncell=40, ng=100, nline=20000, seed=13, lines="synthetic")
    ni = case.gas.ion_ni
    slots = [(iz, ii) for iz in range(1, len(ni) + 1) for ii in range(1, min(iz, int(ni[iz - 1]) - 1) + 1)]
    assert len(slots) >= nrow
    lines = case.lines.copy()
    pick = np.arange(len(lines)) % nrow
    lines["iz"] = np.array([slots[k][0] for k in pick], dtype=np.int16)
    lines["ii"] = np.array([slots[k][1] for k in pick], dtype=np.int16)
    case = dataclasses.replace(case, lines=lines)
    _setup(hot, case)
    _assert_opacity_parity(_gpu_opacity(hot, case), oracle.physical_opacity(case))


def test_physical_opacity_large_grid_matches_oracle(hot, oracle):
    """A grid of more than 2048 shells (not a multiple of the block's 128):
    the forward takes four shells per lane there."""
    case = cases.reference_opacity_case(oracle, ncell=2100, ng=40, nline=8000, seed=17, lines="synthetic")
    _setup(hot, case)
    _assert_opacity_parity(_gpu_opacity(hot, case), oracle.physical_opacity(case))


def test_physical_opacity_full_timestep_size_matches_oracle(hot, oracle):
    """Opacity at the physical-opacity workload's full size (256 shells x 2000
    groups x 5e5 synthetic lines) on the reference's Verner, Sutherland and
    data.ion tables, against the single-threaded oracle (about 2 s)."""
    case = cases.reference_opacity_case(oracle, ncell=256, ng=2000, nline=500_000, seed=2, lines="synthetic")
    _setup(hot, case)
    ref = oracle.physical_opacity(case)
    got = _gpu_opacity(hot, case)
    _assert_opacity_parity(got, ref)
    grey, ross = hot.opacity_means(case.gas.temp, ref["sig"], ref["cap"])
    np.testing.assert_allclose(grey, oracle.planckmean(case.groups.wlinv, case.gas.temp, ref["cap"]), rtol=1e-12)
    np.testing.assert_allclose(ross, oracle.rossmean(case.groups.wlinv, case.gas.temp, ref["sig"], ref["cap"]),
                               rtol=1e-12)


def test_physical_opacity_full_timestep_size_shape_properties(hot):
    case = cases.opacity_case(ncell=256, ng=2000, nline=500_000, seed=2)
    _setup(hot, case)
    got = _gpu_opacity(hot, case)
    assert np.all(np.isfinite(got["cap64"])) and np.all(got["cap64"] >= 0)
    # idempotence: a second call gives bit-identical results
    got2 = _gpu_opacity(hot, case)
    assert np.array_equal(got["cap64"], got2["cap64"])
    assert np.array_equal(got["cap"], got2["cap"])
    # linearity in the line strengths: doubling every gxs doubles the bb part
    bb = hot.physical_opacity(case.gas.temp, case.gas.natom, case.gas.nelec, case.grid.vol, case.gas.mass,
                              case.gas.natomfr, case.gas.oc, case.gas.ginv, nobf=True, noff=True, want_cap64=True)
    lines2 = case.lines.copy()
    lines2["gxs"] = lines2["gxs"] * np.float32(2.0)
    hot.set_atomic_data(case.gas.ion_ni, case.gas.oc.shape[1], lines2, case.bf_ph1, case.bf_ph2, case.ff_gff)
    bb2 = hot.physical_opacity(case.gas.temp, case.gas.natom, case.gas.nelec, case.grid.vol, case.gas.mass,
                               case.gas.natomfr, case.gas.oc, case.gas.ginv, nobf=True, noff=True, want_cap64=True)
    np.testing.assert_allclose(bb2["cap64"], 2.0 * bb["cap64"], rtol=1e-15)


def test_unsorted_lines_rejected(hot):
    from superlite_b200 import SlgError
    case = cases.opacity_case(ncell=8, ng=20, nline=100, seed=4)
    lines = case.lines[::-1].copy()
    with pytest.raises(SlgError):
        hot.set_atomic_data(case.gas.ion_ni, case.gas.oc.shape[1], lines, case.bf_ph1, case.bf_ph2, case.ff_gff)


def test_means_match_oracle(hot, oracle):
    case = cases.opacity_case(ncell=64, ng=300, nline=5000, seed=12)
    _setup(hot, case)
    ref = oracle.physical_opacity(case)
    grey, ross = hot.opacity_means(case.gas.temp, ref["sig"], ref["cap"])
    np.testing.assert_allclose(grey, oracle.planckmean(case.groups.wlinv, case.gas.temp, ref["cap"]), rtol=1e-12)
    np.testing.assert_allclose(ross, oracle.rossmean(case.groups.wlinv, case.gas.temp, ref["sig"], ref["cap"]),
                               rtol=1e-12)


@pytest.mark.parametrize("kind", [1, 2, 3])
def test_analytic_opacity_matches_oracle(hot, oracle, kind):
    from superlite_b200 import workloads as W
    grid = W.homologous_grid(64, 5 * W.PC_DAY)
    groups = W.group_grid(100)
    rho, _ = W.broken_powerlaw_rho(grid)
    temp = np.random.default_rng(kind).uniform(6000, 14000, 64)
    hot.set_groups(groups.wl)
    hot.set_grid(grid.xarr, grid.vxarr, grid.vol, grid.divv)
    kw = dict(kind=kind, capcoef=1e18, captpwr=-1.5, caprpwr=2.0, sigcoef=1e-3, sigtpwr=0.5, sigrpwr=1.0,
              ldisp1=0.3, ldisp2=3.0)
    sig, cap = hot.analytic_opacity(temp, rho, **kw)
    rs, rc = oracle.analytic_opacity(groups.wlinv, temp, rho, **kw)
    np.testing.assert_allclose(sig, rs, rtol=1e-15)
    _assert_float_close(cap, rc, 1)
