"""LTE equation of state (ionsmod.f:160-356, GAS/eos_update.f:20-45).

CPU: known-answer checks of the oracle restatement (charge balance, Saha
ratios, the fully ionised limit, ground-level partition functions, the
reference's "leave nelec untouched" exit).  GPU: slg_saha_eos against the
oracle (nelec, oc within 1e-12 relative, same iteration counts).
"""
import numpy as np
import pytest

from superlite_b200 import workloads as W

KB, ME, H = 1.3806505e-16, 9.1093826e-28, 6.6260693e-27
PI2 = 2.0 * 3.1415926535897932385


def _cells(n=48, seed=1, t_days=10.0):
    rng = np.random.default_rng(seed)
    grid = W.homologous_grid(n, t_days * W.PC_DAY)
    rho, _ = W.broken_powerlaw_rho(grid)
    X = np.zeros((n, W.NELEM))
    X[:, np.array(W.ELEMENTS) - 1] = rng.dirichlet(np.ones(len(W.ELEMENTS)), size=n)
    mass, natom, natomfr = W.composition_state(rho, X, grid.vol)
    T = rng.uniform(6000.0, 14000.0, n)
    return grid, T, natom, natomfr


def _stage_pops(ion, q, oc, natom, vol, natomfr):
    """n_{z,ii} (normalised per element) back from oc = natom fr g1 n / (q vol)."""
    g1 = ion.g1
    n = np.zeros_like(oc)
    for iz in range(oc.shape[0]):
        fr = natomfr[:, iz + 1]
        ok = fr > 0
        for ii in range(oc.shape[1]):
            n[iz, ii, ok] = oc[iz, ii, ok] * q[iz, ii] * vol[ok] / (natom[ok] * fr[ok] * g1[iz, ii])
    return n


def test_partition_function_limits(oracle):
    ion = W.ion_table()
    q_cold = oracle.partition(ion, 50.0)
    for iz in range(ion.nelem):
        ni = ion.ni[iz]
        np.testing.assert_allclose(q_cold[iz, :ni - 1], ion.g1[iz, :ni - 1], rtol=1e-12)
        assert q_cold[iz, ni - 1] == 1.0
    q_hot = oracle.partition(ion, 1e13)  # kT far above every level: q -> sum of the weights
    np.testing.assert_allclose(q_hot[0, 0], ion.glev[0, 0, :ion.nlevel[0, 0]].sum(), rtol=1e-6)


def test_charge_balance_and_saha_ratios(oracle):
    ion = W.ion_table()
    q = oracle.partition(ion, 10000.0)
    grid, T, natom, natomfr = _cells()
    nel, oc, ginv, it = oracle.saha_eos(ion, q, T, natom, grid.vol, natomfr, np.ones(len(T)), acc=1e-14,
                                        noc=W.ION_NI)
    assert (it <= 40).all()
    n = _stage_pops(ion, q, oc, natom, grid.vol, natomfr)
    ne = np.einsum("zsc,s->zc", n, np.arange(W.ION_NI, dtype=float))
    charge = (natomfr[:, 1:].T * ne).sum(axis=0)
    np.testing.assert_allclose(charge, nel, rtol=1e-12)
    ndens = natom / grid.vol
    sahac = (PI2 * ME * KB * T / H ** 2) ** 1.5
    for iz in np.array(W.ELEMENTS) - 1:
        for ii in range(W.ION_NI - 1):
            ratio = n[iz, ii + 1] / n[iz, ii]
            want = 2.0 * sahac / (nel * ndens) * np.exp(-ion.e[iz, ii] / (KB * T)) * q[iz, ii + 1] / q[iz, ii]
            ok = n[iz, ii] > 1e-250
            np.testing.assert_allclose(ratio[ok], want[ok], rtol=1e-10)
    np.testing.assert_array_equal(ginv, 1.0 / np.repeat(ion.g1[:, :, None], len(T), axis=2))


def test_fully_ionised_limit_and_untouched_exit(oracle):
    ion = W.ion_table()
    q = oracle.partition(ion, 10000.0)
    grid, T, natom, natomfr = _cells(n=8)
    hot_T = np.full(8, 3e6)
    nel, *_ = oracle.saha_eos(ion, q, hot_T, natom, grid.vol, natomfr, np.ones(8), acc=1e-12)
    np.testing.assert_allclose(nel, W.ION_NI - 1, rtol=1e-6)
    # converged start value: the first iteration exits and leaves nelec as given
    nel1, *_ = oracle.saha_eos(ion, q, T, natom, grid.vol, natomfr, np.ones(8), acc=1e-14)
    nel2, _, _, it = oracle.saha_eos(ion, q, T, natom, grid.vol, natomfr, nel1, acc=1e-8)
    assert (it == 1).all()
    np.testing.assert_array_equal(nel2, nel1)


@pytest.mark.gpu
@pytest.mark.parametrize("acc,start", [(1e-8, 1.0), (1e-8, 0.05), (1e-14, 1.0)])
def test_gpu_saha_eos_matches_oracle(hot, oracle, acc, start):
    ion = W.ion_table()
    grid, T, natom, natomfr = _cells(n=300, seed=4, t_days=6.0)
    hot.set_groups(W.group_grid(10).wl)
    hot.set_grid(grid.xarr, grid.vxarr, grid.vol, grid.divv)
    q = hot.set_ions(ion, q_temp=float(T[0]))
    q_orc = oracle.partition(ion, float(T[0]))
    np.testing.assert_allclose(q, q_orc, rtol=1e-14)
    nel0 = np.full(len(T), start)
    ng, ocg, gig, itg = hot.saha_eos(T, natom, grid.vol, natomfr, nel0, acc=acc, noc=4)
    no, oco, gio, ito = oracle.saha_eos(ion, q_orc, T, natom, grid.vol, natomfr, nel0, acc=acc, noc=4)
    np.testing.assert_array_equal(itg, ito)
    np.testing.assert_allclose(ng, no, rtol=1e-12)
    np.testing.assert_allclose(ocg, oco, rtol=1e-12, atol=0)
    np.testing.assert_array_equal(gig, gio)
