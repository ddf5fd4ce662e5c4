"""Known-answer tests that pin the CPU oracle (no GPU needed).

The reference ships no golden vectors (its `make check` target names a missing
script and Testsuite/ holds inputs only), so the oracle is pinned by analytic
results of the formulas it restates, by published reference values (Philox
known-answer vectors; hydrogenic photo-ionisation thresholds) and by
conservation laws of the transport.
"""
import math

import numpy as np
import pytest

from superlite_b200 import workloads as W


# ---------------------------------------------------------------- Planck integrals
@pytest.mark.parametrize("mode,tol", [(0, 2e-5), (1, 5e-5), (2, 1e-7), (11, 1e-9)])
def test_specintv_normalised(oracle, mode, tol):
    # groupmod.f:146-272: sum over a grid covering x = 1e-5..400 integrates 15/pi^4 x^3/(e^x-1) = 1
    wl = np.geomspace(1e-7, 1e-1, 8001)[::-1].copy()[::-1]
    wlinv = 1.0 / wl
    tinv = 1.0 / 1e4
    s = oracle.specintv(tinv, wlinv, mode=mode).sum()
    # wavelengths below x=400 are clipped at 300 in the reference; the tail is negligible
    assert abs(s - 1.0) < tol


def test_spectintv_normalised(oracle):
    wl = np.geomspace(1e-7, 1e-1, 8001)
    s = oracle.spectintv(1.0 / 1e4, 1.0 / wl, mode=2).sum()
    assert abs(s - 1.0) < 1e-6


def test_specint0_equals_specintv_element(oracle):
    g = W.group_grid(100)
    for T in (3000.0, 1e4, 5e4):
        ss = oracle.specintv(1.0 / T, g.wlinv)
        lib = oracle.lib()
        s0 = np.array([lib.orc_specint0(1.0 / T, g.wlinv.ctypes.data_as(oracle.dp), ig) for ig in range(1, 101)])
        np.testing.assert_allclose(s0, ss, rtol=1e-13)


def test_specintv_offset_matches_full(oracle):
    g = W.group_grid(200)
    full = oracle.specintv(1 / 8000.0, g.wlinv)
    part = oracle.specintv(1 / 8000.0, g.wlinv, n=17, offset=40)
    assert np.array_equal(part, full[39:56])
    bad = oracle.specintv(1 / 8000.0, g.wlinv, n=17, offset=190)  # ioff+n > ng+1
    assert np.all(bad == -1.0)


# ---------------------------------------------------------------- binary search
def test_binsrch_edges(oracle):
    a = np.array([1.0, 2.0, 4.0, 8.0, 16.0])
    assert oracle.binsrch(1.0, a) == 1
    assert oracle.binsrch(16.0, a) == 4
    assert oracle.binsrch(2.0, a) == 2          # x == arr(k) opens interval k
    assert oracle.binsrch(3.9, a) == 2
    assert oracle.binsrch(0.5, a) == 1          # clamped
    assert oracle.binsrch(0.5, a, True) == 0    # widerange
    assert oracle.binsrch(99.0, a) == 4
    assert oracle.binsrch(99.0, a, True) == 5
    assert oracle.binsrch(float("nan"), a) == -1
    two = np.array([1.0, 3.0])
    assert oracle.binsrch(2.0, two) == 1
    assert oracle.binsrch(0.0, two, True) == 0
    assert oracle.binsrch(5.0, two, True) == 2
    assert oracle.binsrch(5.0, two) == 1


# ---------------------------------------------------------------- random numbers
def test_philox_known_answers(oracle):
    # Philox4x32-10 known-answer vectors published with Random123 (kat_vectors)
    import ctypes as C
    lib = oracle.lib()
    # reach the raw generator through the draw mapping: draw k=0/1 of counter 0
    # exposes words (0,1)/(2,3); check the words via the 52-bit mapping.
    def words(ctr, key):
        # pid = ctr[1] | ctr[2] << 32, stream = ctr[3], k = 2*ctr[0] (+1 for words 2,3)
        pid = ctr[1] | (ctr[2] << 32)
        seed = key[0] | (key[1] << 32)
        d0 = lib.orc_philox_draw(seed, pid, ctr[3], 2 * ctr[0])
        d1 = lib.orc_philox_draw(seed, pid, ctr[3], 2 * ctr[0] + 1)
        return d0, d1

    def expect(w):
        m0 = (w[0] << 20) | (w[1] >> 12)
        m1 = (w[2] << 20) | (w[3] >> 12)
        return (m0 + 0.5) * 2.0 ** -52, (m1 + 0.5) * 2.0 ** -52

    kats = [
        ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
        ((0xffffffff, 0xffffffff, 0xffffffff, 0xffffffff), (0xffffffff, 0xffffffff),
         (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ]
    for ctr, key, w in kats:
        if ctr[0] * 2 + 1 > 0xffffffff:
            continue  # k is 32-bit: counter word 0 = k/2 cannot reach 0xffffffff here
        assert words(ctr, key) == expect(w)


def test_philox_range_and_moments(oracle):
    d = np.array([oracle.philox_draw(123, pid, 0, k) for pid in range(200) for k in range(25)])
    assert d.min() > 0.0 and d.max() < 1.0
    assert abs(d.mean() - 0.5) < 0.01
    assert abs(d.var() - 1 / 12) < 0.005


def test_mzran_range(oracle):
    st = oracle.rnd_init(4, 0)
    v = np.array([oracle.rnd_r(st[1]) for _ in range(20000)])
    assert v.min() > 0.0 and v.max() < 1.0
    assert abs(v.mean() - 0.5) < 0.01


# ---------------------------------------------------------------- bound-free
def test_bfxs_threshold_synthetic(oracle):
    ph1, ph2 = W.synthetic_verner()
    t1 = ph1.reshape(30, 30, 7, 6)  # (ne, nz, is, k)
    for nz, ne in [(6, 6), (8, 5), (26, 26), (14, 12)]:
        ntot = [1, 1, 2, 2, 3, 3, 3, 3, 3, 3, 4, 4, 5, 5, 5, 5, 5, 5, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 7, 7]
        nout = 7 if (nz > 18 and nz == ne) else ntot[ne - 1]
        eth = float(t1[ne - 1, nz - 1, nout - 1, 0])
        assert oracle.bfxs(ph1, ph2, nz, ne, eth * (1 - 1e-6)) == 0.0
        assert oracle.bfxs(ph1, ph2, nz, ne, eth * 1.5) > 0.0
    assert oracle.bfxs(ph1, ph2, 31, 1, 100.0) == 0.0
    assert oracle.bfxs(ph1, ph2, 5, 6, 100.0) == 0.0


def test_bfxs_published_thresholds(oracle):
    # Verner et al. (1996) fits: sigma at threshold of H I is 6.30 Mb, of He II
    # 6.30/Z^2 = 1.58 Mb (hydrogenic), of He I 7.4 Mb.  The reference's
    # data.bf_verner, from the committed fixture tests/golden/atomic_data.npz.
    import cases
    ph1, ph2, _ = cases.atomic_data().tables
    # thresholds are real*4: 13.6 eV is stored as 13.6000004, so probe just above
    assert oracle.bfxs(ph1, ph2, 1, 1, 13.6) == 0.0
    assert oracle.bfxs(ph1, ph2, 1, 1, 13.6001) == pytest.approx(6.30, rel=0.02)
    assert oracle.bfxs(ph1, ph2, 2, 1, 54.4201) == pytest.approx(1.58, rel=0.02)
    assert oracle.bfxs(ph1, ph2, 2, 2, 24.5901) == pytest.approx(7.4, rel=0.05)
    assert oracle.bfxs(ph1, ph2, 1, 1, 13.5) == 0.0


# ---------------------------------------------------------------- physical opacity closed forms
def _single_cell_case(nline=1, ng=10):
    case = W.opacity_case(ncell=2, ng=ng, nline=max(nline, 1), seed=5)
    return case


def test_bb_single_line_closed_form(oracle):
    case = _single_cell_case(nline=1, ng=10)
    ln = case.lines
    r = oracle.physical_opacity(case, nobf=True, noff=True)
    wl0 = float(ln["wl0"][0]) * 1e-8
    g = int(np.searchsorted(case.groups.wl, wl0, side="right"))  # 1-based group
    hc, kb, c = W.PC_H * W.PC_C, W.PC_KB, W.PC_C
    for i in range(2):
        T = case.gas.temp[i]
        hckt = hc / (kb * T)
        wa, wb = case.groups.wl[g - 1], case.groups.wl[g]
        wl = 0.5 * (wa + wb)
        phi = wl * wl / ((wb - wa) * c)
        iz, ii = int(ln["iz"][0]), int(ln["ii"][0])
        ocg = case.gas.oc[iz - 1, ii - 1, i] * case.gas.ginv[iz - 1, ii - 1, i]
        expect = phi * float(ln["gxs"][0]) * ocg * math.exp(-float(ln["chilw"][0]) * hckt) * (1 - math.exp(-hckt / wl))
        got = r["cap64"][i]
        assert got[g - 1] == pytest.approx(expect, rel=1e-13)
        assert np.count_nonzero(got) == 1
        assert r["cap"][i, g - 1] == np.float32(got[g - 1])


def test_ff_bilinear_exact_on_linear_table(oracle):
    case = _single_cell_case(ng=30)
    iu, igg = np.meshgrid(np.arange(1, 82), np.arange(1, 42), indexing="ij")
    gff = 1.0 + 0.01 * iu + 0.002 * igg
    case.ff_gff = np.asfortranarray(gff).ravel(order="F")
    r = oracle.physical_opacity(case, nobb=True, nobf=True)
    hc, kb = W.PC_H * W.PC_C, W.PC_KB
    c1 = 4 * W.PC_E ** 6 / (3 * W.PC_H * W.PC_ME * W.PC_C ** 4) * math.sqrt(2 * math.pi / (3 * W.PC_ME * W.PC_H * W.PC_C))
    g = case.gas
    for i in range(2):
        hckt = hc / (kb * g.temp[i])
        hl = (g.natom[i] / case.grid.vol[i]) ** 2 * g.nelec[i]
        for ig in range(30):
            wl = case.groups.wl[ig]
            u = hckt / wl
            ru = min(max(10 * (math.log10(u) + 4) + 1, 1.0), 80.999999)
            help_ = c1 * math.sqrt(hckt) * (1 - math.exp(-u)) * wl ** 3 * hl
            tot = 0.0
            for iz in range(1, 31):
                fr = g.natomfr[i, iz]
                if fr == 0:
                    continue
                rgg = 5 * (math.log10(iz * iz * W.PC_RYDBERG_CM * hckt) + 4) + 1 if hasattr(W, "PC_RYDBERG_CM") else \
                    5 * (math.log10(iz * iz * 1.0973731534e5 * hckt) + 4) + 1
                rgg = min(max(rgg, 1.0), 40.999999)
                val = 1.0 + 0.01 * ru + 0.002 * rgg
                tot += help_ * val * iz * iz * fr
            assert r["cap64"][i, ig] == pytest.approx(tot, rel=1e-10)


def test_means_of_grey_opacity(oracle):
    g = W.group_grid(300)
    T = np.array([5000.0, 9000.0, 20000.0])
    cap = np.full((3, 300), 2.5, dtype=np.float32)
    grey = oracle.planckmean(g.wlinv, T, cap)
    for k in range(3):
        norm = oracle.specintv(1 / T[k], g.wlinv).sum()
        assert grey[k] == pytest.approx(2.5 * norm, rel=1e-13)
    sig = np.array([0.5, 0.0, 1.0])
    ross = oracle.rossmean(g.wlinv, T, sig, cap)
    for k in range(3):
        norm = oracle.spectintv(1 / T[k], g.wlinv).sum()
        assert ross[k] == pytest.approx((2.5 + sig[k]) / norm, rel=1e-13)


def test_physical_opacity_flags_and_subgroups(oracle):
    case = W.opacity_case(ncell=4, ng=20, nline=500, seed=9)
    r1 = oracle.physical_opacity(case)
    assert r1["flags"] & ~1 == 0  # no negative / NaN / inf
    r2 = oracle.physical_opacity(case, ngs=3, opacmixrossel=0.0)
    # Planck-mixed collapse of 3 sub-groups stays positive and finite
    assert np.all(np.isfinite(r2["cap64"])) and np.all(r2["cap64"] >= 0)


# ---------------------------------------------------------------- grid coefficients
def test_emitgroup_consistent_with_emitprob(oracle):
    import cases
    c = cases.transport_case(oracle, t_days=5.0, npart=200)
    t = c["tables"]
    g = c["groups"]
    # sampled groups follow w_g * kappa_g; check the first-moment of many draws
    ic = 20
    spec = oracle.specintv(t["tempinv"][ic - 1], g.wlinv)
    w = spec * t["cap"][ic - 1].astype(np.float64)
    rs = (np.arange(4000) + 0.5) / 4000
    gs = np.array([oracle.emitgroup(r, ic, g.wlinv, t["tempinv"], t["cap"], t["capgrey"], t["emitprob"]) for r in rs])
    assert gs.min() >= 1 and gs.max() <= g.ng
    cdf = np.cumsum(w) / w.sum()
    emp = np.array([(gs <= k + 1).mean() for k in range(g.ng)])
    assert np.max(np.abs(emp - cdf)) < 0.02


def test_leakage_nonnegative_and_lumping(oracle):
    import cases
    c = cases.transport_case(oracle, t_days=2.0, npart=200)
    ol = c["tables"]["opaclump"]
    assert np.all(ol[:, [0, 1, 6, 7]] >= 0)
    thick = ol[:, 6] > 0
    assert thick.any()
    # speclump = 1/sum of lumped Planck weights <= ... >= 1
    assert np.all(ol[thick, 6] >= 1.0 - 1e-12)


# ---------------------------------------------------------------- transport conservation
def _lab_energy(c):
    """Sum of particle energies after the initial comoving->lab transform (particle_advance.f90:186-195)."""
    prt, isv = c["prt"], c["isv"]
    g = c["grid"]
    t = c["tables"]
    live = isv == 0
    x = prt["x"][live]
    ix = np.clip(np.searchsorted(g.xarr, x, side="right"), 1, g.nx)
    vx = (g.vxarr[ix - 1] * (g.xarr[ix] - x) + g.vxarr[ix] * (x - g.xarr[ix - 1])) / (g.xarr[ix] - g.xarr[ix - 1])
    ig = np.clip(np.searchsorted(c["groups"].wl, prt["wl"][live], side="right"), 1, c["groups"].ng)
    tau = (t["sig"][ix - 1] + t["cap"][ix - 1, ig - 1].astype(np.float64)) * (g.xarr[ix] - g.xarr[ix - 1])
    imc = c["params"].puretran | (tau < c["params"].tauddmc)
    labfact = np.where(imc, 1.0 - vx * prt["mu"][live] / W.PC_C, 1.0)
    return float((prt["e"][live] / labfact).sum())


def test_energy_ledger_pure_imc(oracle):
    import cases
    p = W.TransportParams(puretran=True)
    c = cases.transport_case(oracle, t_days=20.0, npart=3000, params=p)
    e0 = _lab_energy(c)
    tt = oracle.TransportTables(c["grid"], c["groups"], **c["tables"], params=p)
    prt, isv = c["prt"].copy(), c["isv"].copy()
    r = oracle.particle_advance(tt, prt, isv, rngmode=1, seed=1, nthreads=4)
    assert r["ierr"] == 0
    assert r["nflux"] == r["npckt"]          # no census, nothing dies in pure IMC
    assert r["tot_eout"] + r["tot_evelo"] == pytest.approx(e0, rel=1e-11)
    lum, dev, num = oracle.fluxtally(prt, isv, c["groups"].wl)
    assert lum.sum() == pytest.approx(r["tot_eout"], rel=1e-12)
    assert num.sum() == r["nflux"]
    assert np.all(isv == 1)


def test_optically_thin_limit(oracle):
    import cases
    p = W.TransportParams(puretran=True)
    c = cases.transport_case(oracle, t_days=30.0, npart=2000, params=p)
    c["tables"]["cap"][:] = 0.0
    c["tables"]["sig"][:] = 0.0
    e0 = _lab_energy(c)
    tt = oracle.TransportTables(c["grid"], c["groups"], **c["tables"], params=p)
    prt, isv = c["prt"].copy(), c["isv"].copy()
    r = oracle.particle_advance(tt, prt, isv, rngmode=1, seed=2, nthreads=2)
    assert r["nflux"] == r["npckt"] == 2000
    assert r["tot_evelo"] == 0.0
    assert r["tot_eout"] == pytest.approx(e0, rel=1e-13)


def test_ddmc_energy_ledger_with_losses(oracle):
    import cases
    c = cases.transport_case(oracle, t_days=4.0, npart=1500)
    e0 = _lab_energy(c)
    tt = oracle.TransportTables(c["grid"], c["groups"], **c["tables"], params=c["params"])
    prt, isv = c["prt"].copy(), c["isv"].copy()
    r = oracle.particle_advance(tt, prt, isv, rngmode=1, seed=3, nthreads=4)
    assert r["ierr"] == 0 and r["nstepddmc"] > 0
    dead_e = 0.0  # dead particles leave the ledger; bound the imbalance by it
    assert r["tot_eout"] + r["tot_evelo"] <= e0 * (1 + 1e-9)
    assert r["tot_eout"] + r["tot_evelo"] > 0.5 * e0


def _early_thick_model(oracle, npart):
    """Model 121 of the batched workload (W.analytic_batch(128, seed=4)): t = 1.01 d,
    225 shells, analytic grey opacity, 195 DDMC shells and IMC shells sandwiched
    between DDMC shells near the photosphere."""
    b = W.analytic_batch(nmodel=128, seed=4)
    m = 121
    co = np.concatenate([[0], np.cumsum(b.nx)])
    nx = int(b.nx[m])
    grid = W.homologous_grid(nx, float(b.t_days[m]) * W.PC_DAY)
    temp, rho = b.temp[co[m]:co[m + 1]], b.rho[co[m]:co[m + 1]]
    groups = b.groups
    sig, cap = W.analytic_grey(grid, temp, rho, groups.ng)
    tinv = 1.0 / temp
    capgrey = oracle.planckmean(groups.wlinv, temp, cap)
    params = W.TransportParams()
    ol = oracle.leakage_opacity11(grid, groups.wlinv, tinv, sig, cap)
    ep = oracle.emission_probability(groups.wlinv, tinv, cap, capgrey, groups.nep, groups.nepg)
    prt, isv, _, _, _ = oracle.make_source_particles(grid, groups, temp, 1e42, npart)
    tables = dict(tempinv=tinv, sig=sig, capgrey=capgrey, emitprob=ep, opaclump=ol, cap=cap)
    return dict(grid=grid, groups=groups, tables=tables, prt=prt, isv=isv, params=params, b=b, m=m)


def test_energy_ledger_early_thick_model(oracle):
    """The t = 1 d model gains energy in the reference's scheme.

    The IMC->DDMC interface reflections (transport11.f90:382-388 outer face,
    :436-444 inner face) resample the direction in the comoving frame and move
    it to the lab frame, but leave the lab-frame energy as it was.  Where an
    IMC shell lies between two DDMC shells, the outward net flux makes
    outer-face reflections outnumber inner-face ones, so reflected particles
    carry more comoving energy than they came with; the next effective
    scattering (transport11.f90:312-320) turns that into lab-frame energy.  A
    particle trapped there for thousands of events compounds the gain.  The
    ledger itself still closes exactly: every change of e is booked in
    tot_evelo (here tot_evelo < 0, the "fluid" gives energy).

    Expected values (Philox seed 3, 3000 particles): escaped / emitted lab
    energy 1.037, about 3 % of escaping particles with more than twice their
    initial energy, the largest gain about 1.4e3.  Other seeds give 0.55-0.62
    with largest gains 15-40: the sum is heavy-tailed.
    """
    c = _early_thick_model(oracle, 3000)
    tau = c["tables"]["cap"][:, 0] * np.diff(c["grid"].xarr)
    ddmc = tau >= c["params"].tauddmc
    # runs of IMC shells with DDMC shells on both sides (shells 194-195 and 197-198 here)
    edges = np.flatnonzero(np.diff(ddmc.astype(np.int8)))
    inner_runs = [(a + 1, b) for a, b in zip(edges[:-1], edges[1:]) if ddmc[a] and not ddmc[a + 1]]
    assert len(inner_runs) >= 2
    e0 = _lab_energy(c)
    tt = oracle.TransportTables(c["grid"], c["groups"], **c["tables"], params=c["params"])
    prt, isv = c["prt"].copy(), c["isv"].copy()
    ein = prt["e"].copy()
    r = oracle.particle_advance(tt, prt, isv, rngmode=1, seed=3, nthreads=4)
    assert r["ierr"] == 0 and r["nflux"] == r["npckt"] == 3000
    assert r["tot_eout"] + r["tot_evelo"] == pytest.approx(e0, rel=1e-11)
    assert 0.95 < r["tot_eout"] / e0 < 1.15
    assert r["tot_evelo"] < 0.0
    gain = prt["e"][isv == 0] / ein[isv == 0]
    assert 0.015 < (gain > 2.0).mean() < 0.06
    assert gain.max() > 300.0


def test_atomic_fixture_is_the_reference_data():
    """The committed atomic-data fixture holds the reference's tables: published
    ionisation potentials of data.ion (H I 13.598 eV, Fe I 7.902 eV, Fe II
    16.19 eV), ground-level weights (H I 2, C I 1), a positive Sutherland
    table, and real lines packed as read_bbxs_data.f does."""
    import cases
    A = cases.atomic_data()
    ev = A.ion.e / W.PC_EV
    assert ev[0, 0] == pytest.approx(13.598, abs=2e-3)
    assert ev[25, 0] == pytest.approx(7.902, abs=2e-3) and ev[25, 1] == pytest.approx(16.19, abs=1e-2)
    assert A.ion.glev[0, 0, 0] == 2.0 and A.ion.glev[5, 0, 0] == 1.0
    assert list(A.ion.ni[[0, 1, 25]]) == [2, 3, 10]
    gff = A.ff_gff.reshape(41, 81)  # Fortran ff_gff(81,41): u fastest
    assert gff.shape == (41, 81) and np.all(np.isfinite(gff)) and np.all(gff > 0)
    ln = A.lines
    assert len(ln) == 16000 and np.all(np.diff(ln["wl0"]) >= 0)
    assert set(np.unique(ln["iz"])) <= set(W.ELEMENTS) and set(np.unique(ln["ii"])) <= {1, 2, 3, 4}
    assert np.all(ln["gxs"] > 0) and ln["wl0"].min() >= 1000.0 and ln["wl0"].max() <= 32000.0


def test_mzran_mode_reproducible(oracle):
    import cases
    c = cases.transport_case(oracle, t_days=15.0, npart=800)
    tt = oracle.TransportTables(c["grid"], c["groups"], **c["tables"], params=c["params"])
    outs = []
    for _ in range(2):
        st = oracle.rnd_init(3, 0)
        prt, isv = c["prt"].copy(), c["isv"].copy()
        outs.append(oracle.particle_advance(tt, prt, isv, rngmode=0, nthreads=3, rnd_states=st))
    assert outs[0]["nstepimc"] == outs[1]["nstepimc"]
    assert np.array_equal(outs[0]["tally"], outs[1]["tally"])


def test_sourcetally_counts(oracle):
    import cases
    c = cases.transport_case(oracle, t_days=10.0, npart=3000)
    rc, en, num = oracle.sourcetally(c["prt"], c["isv"], c["grid"], c["groups"])
    assert rc == 0
    assert num.sum() == 3000
    assert en.sum() == pytest.approx(c["prt"]["e"].sum(), rel=1e-12)
