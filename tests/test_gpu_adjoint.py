"""Hand-written adjoint of the opacity build (slg_dev_opacity_grad_backward)
against central finite differences of its own forward.

L = sum of randomly weighted outputs (group opacities, Thomson opacity,
Planck / Rosseland means, leakage opacities).  For random directions v in
temperature, density and mass fractions, the directional derivative from the
adjoint, grad(L) . v, must match (L(x + h v) - L(x - h v)) / 2h within 1e-6
relative.  Mass-fraction directions keep absent elements at zero (the
reference stops on negative fractions).
"""
import numpy as np
import pytest
import torch

from superlite_b200 import HotPath
from superlite_b200 import workloads as W
from superlite_b200.differentiable import DifferentiableOpacity

pytestmark = pytest.mark.gpu

RTOL = 1e-6


def _setup(nc=24, ng=120, nline=20000, seed=3, t_days=8.0, atomic=None):
    """atomic=None: synthetic tables and ion data; else a workloads.AtomicData
    (the reference's Verner, Sutherland and data.ion tables)."""
    case = W.opacity_case(ncell=nc, ng=ng, nline=nline, seed=seed, t_days=t_days,
                          tables=None if atomic is None else atomic.tables)
    ion = W.ion_table() if atomic is None else atomic.ion
    hot = HotPath(0)
    hot.set_groups(case.groups.wl)
    hot.set_grid(case.grid.xarr, case.grid.vxarr, case.grid.vol, case.grid.divv)
    g = case.gas
    nstage = g.oc.shape[1] if atomic is None else ion.nstage - 1
    hot.set_atomic_data(np.ascontiguousarray(ion.ni, dtype=np.int32), nstage, case.lines, case.bf_ph1, case.bf_ph2,
                        case.ff_gff)
    amass = [W.ELEM_MASS.get(z, 2.0 * z) for z in range(1, W.NELEM + 1)]
    D = DifferentiableOpacity(hot, ion, q_temp=float(g.temp[0]), elem_mass=amass)
    dev = D.device
    T = torch.tensor(g.temp, dtype=torch.float64, device=dev)
    R = torch.tensor(g.rho, dtype=torch.float64, device=dev)
    X = torch.tensor(g.massfr, dtype=torch.float64, device=dev)
    return hot, D, case, T, R, X


def _loss_weights(outs, seed):
    gen = torch.Generator(device=outs[0].device).manual_seed(seed)
    ws = []
    for o in outs:
        w = torch.randn(o.shape, generator=gen, device=o.device, dtype=torch.float64)
        if o.dim() == 2 and o.shape[1] == 11:  # opaclump: scale each row by its own size
            w = w / (o.abs().mean(dim=0, keepdim=True) + 1e-300)
        else:
            w = w / (o.abs().mean() + 1e-300)
        ws.append(w / o.numel())
    ws[4][:, [2, 3, 4, 5, 8, 9]] = 0.0  # rows without a gradient (zero or integer)
    return ws


def _L(D, ws, T, R, X):
    outs = D.opacity(T, R, X)
    return sum((w * o).sum() for w, o in zip(ws, outs))


def _check_central_differences(hot, D, T, R, X, which, ntrial=3):
    with torch.no_grad():
        outs = D.opacity(T, R, X)
    ws = _loss_weights(outs, seed=7)
    Tg, Rg, Xg = T.clone().requires_grad_(), R.clone().requires_grad_(), X.clone().requires_grad_()
    L = _L(D, ws, Tg, Rg, Xg)
    L.backward()
    grads = {"temp": Tg.grad, "rho": Rg.grad, "massfr": Xg.grad}
    gen = torch.Generator(device=T.device).manual_seed(11)
    base = {"temp": T, "rho": R, "massfr": X}[which]
    h = 1e-6
    for trial in range(ntrial):
        v = torch.randn(base.shape, generator=gen, device=T.device, dtype=torch.float64) * base
        if which == "massfr":
            v = v * (X > 0)
        ad = float((grads[which] * v).sum())

        def at(s):
            args = {"temp": T, "rho": R, "massfr": X}
            args[which] = base + s * h * v
            with torch.no_grad():
                return float(_L(D, ws, args["temp"], args["rho"], args["massfr"]))

        fd = (at(1.0) - at(-1.0)) / (2.0 * h)
        assert ad == pytest.approx(fd, rel=RTOL), (which, trial, ad, fd)


@pytest.mark.parametrize("tables", ["synthetic", "reference"])
@pytest.mark.parametrize("which", ["temp", "rho", "massfr"])
def test_adjoint_matches_central_differences(which, tables):
    import cases
    hot, D, case, T, R, X = _setup(atomic=cases.atomic_data() if tables == "reference" else None)
    _check_central_differences(hot, D, T, R, X, which)
    hot.close()


@pytest.mark.parametrize("which", ["temp", "massfr"])
def test_adjoint_large_grid_matches_central_differences(which):
    """A grid large enough (population rows referenced by lines x shells >=
    32768, kBwdGlobalAccMin in csrc/opacity.cu) that the adjoint accumulates
    d/d(population) by global reductions instead of shared-memory atomics."""
    hot, D, case, T, R, X = _setup(nc=1024, ng=60, nline=20000, seed=9)
    rows = len(set(zip(case.lines["iz"].tolist(), case.lines["ii"].tolist())))
    assert rows * 1024 >= 32768, rows
    _check_central_differences(hot, D, T, R, X, which, ntrial=2)
    hot.close()


def test_forward_equals_standard_path():
    """The differentiable forward runs the same kernels as slg_saha_eos +
    slg_physical_opacity: the same nelec, opacities and Thomson opacity."""
    hot, D, case, T, R, X = _setup(nc=16, ng=80)
    with torch.no_grad():
        cap, sig, grey, ross, ol = D.opacity(T, R, X)
    nelec = D.nelec.cpu().numpy()
    mass, natom, natomfr = W.composition_state(case.gas.rho, case.gas.massfr, case.grid.vol)
    nel, oc, ginv, it = hot.saha_eos(case.gas.temp, natom, case.grid.vol, natomfr, np.ones(16), acc=1e-14, noc=4)
    np.testing.assert_allclose(nel, nelec, rtol=1e-12)
    op = hot.physical_opacity(case.gas.temp, natom, nel, case.grid.vol, mass, natomfr, oc, ginv)
    np.testing.assert_allclose(cap.cpu().numpy().astype(np.float32), op["cap"], rtol=2e-7)
    np.testing.assert_allclose(sig.cpu().numpy(), op["sig"], rtol=1e-12)
    hot.close()


@pytest.mark.parametrize("which", ["temp", "rho", "massfr"])
def test_adjoint_matches_oracle_central_differences(oracle, which):
    """The FP64 reference gradient: central differences of the oracle's
    forward (the C++ restatement of the Fortran: composition, ions_solve_eos
    with the partition functions frozen at one temperature, physical_opacity)
    against the GPU adjoint, for L = <w_cap, cap> + <w_sig, sig>, within 1e-6
    relative along random directions."""
    import dataclasses
    nc, ng = 12, 80
    hot, D, case, T, R, X = _setup(nc=nc, ng=ng, nline=5000, seed=5)
    g = case.gas
    ion = W.ion_table()
    q = oracle.partition(ion, float(g.temp[0]))
    gen = np.random.default_rng(17)
    wcap = gen.standard_normal((nc, ng))
    wsig = gen.standard_normal(nc)

    def L_oracle(Tn, Rn, Xn):
        mass, natom, natomfr = W.composition_state(Rn, Xn, case.grid.vol)
        nel, oc, ginv, it = oracle.saha_eos(ion, q, Tn, natom, case.grid.vol, natomfr, np.ones(nc), acc=1e-14,
                                            noc=g.oc.shape[1])
        gas = dataclasses.replace(g, temp=Tn, mass=mass, rho=Rn, natom=natom, nelec=nel, natomfr=natomfr,
                                  massfr=Xn, oc=oc, ginv=ginv)
        r = oracle.physical_opacity(dataclasses.replace(case, gas=gas))
        return r["cap64"], r["sig"]

    cap0, sig0 = L_oracle(g.temp, g.rho, g.massfr)
    scale_c = 1.0 / (np.abs(cap0).mean() * cap0.size)
    scale_s = 1.0 / (np.abs(sig0).mean() * sig0.size)
    Tg, Rg, Xg = T.clone().requires_grad_(), R.clone().requires_grad_(), X.clone().requires_grad_()
    cap, sig, grey, ross, ol = D.opacity(Tg, Rg, Xg)
    np.testing.assert_allclose(cap.detach().cpu().numpy(), cap0, rtol=1e-10)
    np.testing.assert_allclose(sig.detach().cpu().numpy(), sig0, rtol=1e-10)
    wc = torch.tensor(wcap * scale_c, device=T.device)
    wsg = torch.tensor(wsig * scale_s, device=T.device)
    ((wc * cap).sum() + (wsg * sig).sum()).backward()
    grad = {"temp": Tg.grad, "rho": Rg.grad, "massfr": Xg.grad}[which].cpu().numpy()
    base = {"temp": g.temp, "rho": g.rho, "massfr": g.massfr}[which]
    h = 1e-6
    for trial in range(2):
        v = gen.standard_normal(base.shape) * base
        ad = float((grad * v).sum())

        def at(s):
            args = {"temp": g.temp, "rho": g.rho, "massfr": g.massfr}
            args[which] = base + s * h * v
            c, sg = L_oracle(args["temp"], args["rho"], args["massfr"])
            return float((wcap * scale_c * c).sum() + (wsig * scale_s * sg).sum())

        fd = (at(1.0) - at(-1.0)) / (2.0 * h)
        assert ad == pytest.approx(fd, rel=RTOL), (which, trial, ad, fd)
    hot.close()
