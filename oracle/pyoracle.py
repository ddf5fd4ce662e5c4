"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py as the checker.  The product (superlite_b200)
never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

PACKET_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("mu", "<f8"),
                         ("om", "<f8"), ("e", "<f8"), ("e0", "<f8"), ("wl", "<f8")])

dp = C.POINTER(C.c_double)
fp = C.POINTER(C.c_float)
ip = C.POINTER(C.c_int32)


class OpacIn(C.Structure):
    _fields_ = [("ncell", C.c_int32), ("ng", C.c_int32), ("ngs", C.c_int32), ("nelem", C.c_int32),
                ("nstage", C.c_int32), ("grp_wl", dp), ("temp", dp), ("natom", dp), ("nelec", dp),
                ("vol", dp), ("mass", dp), ("natomfr", dp), ("ion_ni", ip), ("oc", dp), ("ginv", dp),
                ("nline", C.c_int64), ("bb", C.c_void_p), ("bf_ph1", fp), ("bf_ph2", fp),
                ("ff_gff", dp), ("nobb", C.c_int32), ("nobf", C.c_int32), ("noff", C.c_int32),
                ("nothmson", C.c_int32), ("opacmixrossel", C.c_double)]


class TrnIn(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ng", C.c_int32), ("nep", C.c_int32), ("nepg", C.c_int32),
                ("xarr", dp), ("vxarr", dp), ("divv", dp), ("wl", dp), ("wlinv", dp),
                ("tempinv", dp), ("sig", dp), ("capgrey", dp), ("emitprob", dp), ("opaclump", dp),
                ("cap", fp), ("tauddmc", C.c_double), ("taulump", C.c_double),
                ("puretran", C.c_int32), ("noampfact", C.c_int32), ("errorfatal", C.c_int32),
                ("thm_aniso", C.c_int32), ("dogrdtally", C.c_int32), ("max_steps", C.c_int64)]


class TrnOut(C.Structure):
    _fields_ = [("tally", dp), ("jrad", dp), ("eamp", dp), ("methodswap", ip),
                ("tot_evelo", C.c_double), ("tot_eout", C.c_double), ("tot_sflux", C.c_double),
                ("npckt", C.c_int64), ("nflux", C.c_int64), ("nstepimc", C.c_int64),
                ("nstepddmc", C.c_int64), ("nmethodswap", C.c_int64), ("nstepmax", C.c_int64),
                ("ndist", C.c_int64 * 11), ("nposwarn", C.c_int64), ("ierr", C.c_int32),
                ("ierr_part", C.c_int32)]


class OrcIon(C.Structure):
    _fields_ = [("nelem", C.c_int32), ("nstage", C.c_int32), ("ni", C.c_void_p), ("e", C.c_void_p),
                ("q", C.c_void_p), ("g1", C.c_void_p)]


def _ptr(a, t):
    if a is None:
        return None
    return a.ctypes.data_as(t)


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_specint0.restype = C.c_double
        L.orc_specint0.argtypes = [C.c_double, dp, C.c_int]
        L.orc_dopspeccalc.restype = C.c_double
        L.orc_dopspeccalc.argtypes = [C.c_double, dp, C.c_int]
        L.orc_specintv.argtypes = [C.c_double, dp, C.c_int, C.c_int, C.c_int, C.c_int, dp]
        L.orc_spectintv.argtypes = [C.c_double, dp, C.c_int, C.c_int, C.c_int, C.c_int, dp]
        L.orc_planck.restype = C.c_double
        L.orc_planck.argtypes = [C.c_double, C.c_double]
        L.orc_binsrch.restype = C.c_int
        L.orc_binsrch.argtypes = [C.c_double, dp, C.c_int, C.c_int]
        L.orc_bfxs.restype = C.c_double
        L.orc_bfxs.argtypes = [fp, fp, C.c_int, C.c_int, C.c_double]
        L.orc_physical_opacity.restype = C.c_int
        L.orc_physical_opacity.argtypes = [C.POINTER(OpacIn), dp, fp, fp, dp]
        L.orc_analytic_opacity.argtypes = [C.c_int, C.c_int, dp, dp, dp, C.c_int] + [C.c_double] * 8 + [dp, fp]
        L.orc_opacity_planckmean.argtypes = [C.c_int, C.c_int, dp, dp, fp, dp]
        L.orc_opacity_rossmean.argtypes = [C.c_int, C.c_int, dp, dp, dp, fp, dp]
        L.orc_leakage_opacity11.argtypes = [C.c_int, C.c_int, dp, dp, dp, dp, dp, fp, fp, dp,
                                            C.c_double, C.c_double, dp]
        L.orc_emission_probability.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, dp, fp, dp, dp, dp]
        L.orc_emitgroup.restype = C.c_int
        L.orc_emitgroup.argtypes = [C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, dp, fp, dp, dp, dp]
        L.orc_rnd_init.argtypes = [C.c_int, C.c_int, C.c_void_p]
        L.orc_rnd_r.restype = C.c_double
        L.orc_rnd_r.argtypes = [C.c_void_p]
        L.orc_philox_draw.restype = C.c_double
        L.orc_philox_draw.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32]
        L.orc_particle_advance.restype = C.c_int
        L.orc_particle_advance.argtypes = [C.POINTER(TrnIn), C.c_void_p, ip, C.c_int64, C.c_int,
                                           C.c_uint64, C.c_int, C.c_void_p, C.POINTER(TrnOut),
                                           C.POINTER(C.c_uint64), ip]
        L.orc_fluxtally.argtypes = [C.c_int64, C.c_void_p, ip, C.c_int, dp, dp, dp, ip]
        L.orc_sourcetally.restype = C.c_int
        L.orc_sourcetally.argtypes = [C.c_int64, C.c_void_p, ip, C.c_int, C.c_int, dp, dp, dp, ip]
        L.orc_sourceenergy.argtypes = [C.c_int, dp, dp, C.c_double, dp, dp]
        L.orc_sourcenumbers.restype = C.c_int64
        L.orc_sourcenumbers.argtypes = [C.c_int, dp, C.c_double, C.c_int64, C.c_int64, ip]
        L.orc_interior_source.restype = C.c_int
        L.orc_interior_source.argtypes = [C.c_int, C.c_int, dp, dp, dp, dp, dp, C.c_double, ip,
                                          C.c_int64, C.c_void_p, ip, C.c_void_p, C.c_int, C.c_uint64]
        L.orc_partition.argtypes = [C.c_int, C.c_int, C.c_int, ip, ip, dp, dp, C.c_double, dp]
        L.orc_saha_eos.restype = C.c_int
        L.orc_saha_eos.argtypes = [C.POINTER(OrcIon), C.c_int, dp, dp, dp, dp, C.c_double, dp, C.c_int32, dp, dp, ip]
        _LIB = L
    return _LIB


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


# ---------------------------------------------------------------- groups
def specintv(tempinv, wlinv, n=None, offset=1, mode=0):
    wlinv = f64(wlinv)
    ng = len(wlinv) - 1
    n = ng if n is None else n
    ss = np.zeros(n)
    lib().orc_specintv(tempinv, _ptr(wlinv, dp), ng, n, offset, mode, _ptr(ss, dp))
    return ss


def spectintv(tempinv, wlinv, n=None, offset=1, mode=0):
    wlinv = f64(wlinv)
    ng = len(wlinv) - 1
    n = ng if n is None else n
    ss = np.zeros(n)
    lib().orc_spectintv(tempinv, _ptr(wlinv, dp), ng, n, offset, mode, _ptr(ss, dp))
    return ss


def binsrch(x, arr, widerange=False):
    arr = f64(arr)
    return lib().orc_binsrch(float(x), _ptr(arr, dp), len(arr), int(widerange))


def bfxs(ph1, ph2, nz, ne, e):
    return lib().orc_bfxs(_ptr(f32(ph1), fp), _ptr(f32(ph2), fp), nz, ne, float(e))


# ---------------------------------------------------------------- opacity
def physical_opacity(case, ngs=1, nobb=False, nobf=False, noff=False, nothmson=False,
                     opacmixrossel=0.0):
    """Returns dict(sig, cap (ncell,ng) f32, emiss, cap64 (ncell,ng) f64, flags)."""
    g = case.gas
    nc, ng = case.grid.nx, case.groups.ng
    keep = dict(wl=f64(case.groups.wl), temp=f64(g.temp), natom=f64(g.natom), nelec=f64(g.nelec),
                vol=f64(case.grid.vol), mass=f64(g.mass), natomfr=f64(g.natomfr),
                ion_ni=np.ascontiguousarray(g.ion_ni, dtype=np.int32), oc=f64(g.oc), ginv=f64(g.ginv),
                bb=np.ascontiguousarray(case.lines), ph1=f32(case.bf_ph1), ph2=f32(case.bf_ph2),
                gff=f64(case.ff_gff))
    oin = OpacIn(nc, ng, ngs, 30, g.oc.shape[1], _ptr(keep["wl"], dp), _ptr(keep["temp"], dp),
                 _ptr(keep["natom"], dp), _ptr(keep["nelec"], dp), _ptr(keep["vol"], dp),
                 _ptr(keep["mass"], dp), _ptr(keep["natomfr"], dp), _ptr(keep["ion_ni"], ip),
                 _ptr(keep["oc"], dp), _ptr(keep["ginv"], dp), len(keep["bb"]),
                 keep["bb"].ctypes.data_as(C.c_void_p), _ptr(keep["ph1"], fp), _ptr(keep["ph2"], fp),
                 _ptr(keep["gff"], dp), int(nobb), int(nobf), int(noff), int(nothmson),
                 float(opacmixrossel))
    sig = np.zeros(nc)
    cap = np.zeros((nc, ng), dtype=np.float32)
    emiss = np.zeros((nc, ng), dtype=np.float32)
    cap64 = np.zeros((ng, nc))
    flags = lib().orc_physical_opacity(C.byref(oin), _ptr(sig, dp), _ptr(cap, fp), _ptr(emiss, fp),
                                       _ptr(cap64, dp))
    return dict(sig=sig, cap=cap, emiss=emiss, cap64=np.ascontiguousarray(cap64.T), flags=flags)


def planckmean(wlinv, temp, cap):
    nc, ng = cap.shape
    out = np.zeros(nc)
    lib().orc_opacity_planckmean(nc, ng, _ptr(f64(wlinv), dp), _ptr(f64(temp), dp),
                                 _ptr(f32(cap), fp), _ptr(out, dp))
    return out


def rossmean(wlinv, temp, sig, cap):
    nc, ng = cap.shape
    out = np.zeros(nc)
    lib().orc_opacity_rossmean(nc, ng, _ptr(f64(wlinv), dp), _ptr(f64(temp), dp), _ptr(f64(sig), dp),
                               _ptr(f32(cap), fp), _ptr(out, dp))
    return out


def analytic_opacity(wlinv, temp, rho, kind=1, capcoef=1e18, captpwr=-1.5, caprpwr=2.0,
                     sigcoef=0.0, sigtpwr=0.0, sigrpwr=0.0, ldisp1=1.0, ldisp2=1.0):
    nc = len(temp)
    ng = len(wlinv) - 1
    sig = np.zeros(nc)
    cap = np.zeros((nc, ng), dtype=np.float32)
    lib().orc_analytic_opacity(nc, ng, _ptr(f64(wlinv), dp), _ptr(f64(temp), dp), _ptr(f64(rho), dp),
                               kind, capcoef, captpwr, caprpwr, sigcoef, sigtpwr, sigrpwr, ldisp1,
                               ldisp2, _ptr(sig, dp), _ptr(cap, fp))
    return sig, cap


# ---------------------------------------------------------------- grid coefficients
def leakage_opacity11(grid, wlinv, tempinv, sig, cap, capemit=None, tauddmc=5.0, taulump=10.0):
    nx, ng = cap.shape
    ol = np.zeros((nx, 11))
    ce = None if capemit is None else f32(capemit)
    lib().orc_leakage_opacity11(nx, ng, _ptr(f64(grid.xarr), dp), _ptr(f64(grid.vol), dp),
                                _ptr(f64(grid.divv), dp), _ptr(f64(tempinv), dp), _ptr(f64(sig), dp),
                                _ptr(f32(cap), fp), _ptr(ce, fp) if ce is not None else None,
                                _ptr(f64(wlinv), dp), tauddmc, taulump, _ptr(ol, dp))
    return ol


def emission_probability(wlinv, tempinv, cap, capgrey, nep, nepg):
    nx, ng = cap.shape
    ep = np.zeros((nx, nep))
    lib().orc_emission_probability(nx, ng, nep, nepg, _ptr(f64(tempinv), dp), _ptr(f32(cap), fp),
                                   _ptr(f64(capgrey), dp), _ptr(f64(wlinv), dp), _ptr(ep, dp))
    return ep


def emitgroup(r, ic, wlinv, tempinv, cap, capgrey, emitprob):
    nx, ng = cap.shape
    nep = emitprob.shape[1]
    nepg = int(np.ceil(ng / (nep + 1.0)))
    return lib().orc_emitgroup(float(r), ic, ng, nep, nepg, _ptr(f64(tempinv), dp), _ptr(f32(cap), fp),
                               _ptr(f64(capgrey), dp), _ptr(f64(emitprob), dp), _ptr(f64(wlinv), dp))


# ---------------------------------------------------------------- rng
def rnd_init(n, ioffset=0):
    st = np.zeros((n, 4), dtype=np.int32)
    lib().orc_rnd_init(n, ioffset, st.ctypes.data_as(C.c_void_p))
    return st


def rnd_r(state):
    return lib().orc_rnd_r(state.ctypes.data_as(C.c_void_p))


def philox_draw(seed, pid, stream, k):
    return lib().orc_philox_draw(seed, pid, stream, k)


# ---------------------------------------------------------------- transport
class TransportTables:
    """Everything particle_advance reads, in the reference's layouts."""

    def __init__(self, grid, groups, tempinv, sig, cap, capgrey, emitprob, opaclump, params):
        self.grid, self.groups = grid, groups
        self.arrays = dict(xarr=f64(grid.xarr), vxarr=f64(grid.vxarr), divv=f64(grid.divv),
                           wl=f64(groups.wl), wlinv=f64(groups.wlinv), tempinv=f64(tempinv),
                           sig=f64(sig), capgrey=f64(capgrey), emitprob=f64(emitprob),
                           opaclump=f64(opaclump), cap=f32(cap))
        self.params = params
        a = self.arrays
        self.cin = TrnIn(grid.nx, groups.ng, groups.nep, groups.nepg, _ptr(a["xarr"], dp),
                         _ptr(a["vxarr"], dp), _ptr(a["divv"], dp), _ptr(a["wl"], dp), _ptr(a["wlinv"], dp),
                         _ptr(a["tempinv"], dp), _ptr(a["sig"], dp), _ptr(a["capgrey"], dp),
                         _ptr(a["emitprob"], dp), _ptr(a["opaclump"], dp), _ptr(a["cap"], fp),
                         params.tauddmc, params.taulump, int(params.puretran), int(params.noampfact),
                         int(params.errorfatal), int(params.thm_aniso), int(params.dogrdtally),
                         int(params.max_steps))


def particle_advance(tt, prt, isvacant, rngmode=1, seed=0, nthreads=1, rnd_states=None, trace=False):
    """Runs orc_particle_advance in place on prt / isvacant.  Returns a dict of tallies."""
    nx, ng = tt.grid.nx, tt.groups.ng
    assert prt.dtype == PACKET_DTYPE and prt.flags.c_contiguous
    assert isvacant.dtype == np.int32
    tally, jrad, eamp = np.zeros(nx), np.zeros((nx, ng)), np.zeros(nx)
    mswap = np.zeros(nx, dtype=np.int32)
    out = TrnOut(_ptr(tally, dp), _ptr(jrad, dp), _ptr(eamp, dp), _ptr(mswap, ip), 0.0, 0.0, 0.0)
    th = np.zeros(len(prt), dtype=np.uint64) if trace else None
    tn = np.zeros(len(prt), dtype=np.int32) if trace else None
    if rngmode == 0:
        assert rnd_states is not None and rnd_states.shape == (nthreads, 4)
    rc = lib().orc_particle_advance(C.byref(tt.cin), prt.ctypes.data_as(C.c_void_p), _ptr(isvacant, ip),
                                    len(prt), rngmode, seed, nthreads,
                                    rnd_states.ctypes.data_as(C.c_void_p) if rnd_states is not None else None,
                                    C.byref(out), th.ctypes.data_as(C.POINTER(C.c_uint64)) if trace else None,
                                    _ptr(tn, ip) if trace else None)
    res = dict(rc=rc, tally=tally, jrad=jrad, eamp=eamp, methodswap=mswap, tot_evelo=out.tot_evelo,
               tot_eout=out.tot_eout, tot_sflux=out.tot_sflux, npckt=out.npckt, nflux=out.nflux,
               nstepimc=out.nstepimc, nstepddmc=out.nstepddmc, nmethodswap=out.nmethodswap,
               nstepmax=out.nstepmax, ndist=np.array(list(out.ndist)), nposwarn=out.nposwarn,
               ierr=out.ierr, ierr_part=out.ierr_part)
    if trace:
        res["trace_hash"], res["trace_nstep"] = th, tn
    return res


def fluxtally(prt, isvacant, flx_wl):
    ng = len(flx_wl) - 1
    lum, dev, num = np.zeros(ng), np.zeros(ng), np.zeros(ng, dtype=np.int32)
    lib().orc_fluxtally(len(prt), prt.ctypes.data_as(C.c_void_p), _ptr(isvacant, ip), ng,
                        _ptr(f64(flx_wl), dp), _ptr(lum, dp), _ptr(dev, dp), _ptr(num, ip))
    return lum, dev, num


def sourcetally(prt, isvacant, grid, groups):
    nx, ng = grid.nx, groups.ng
    en = np.zeros((ng, nx))
    num = np.zeros((ng, nx), dtype=np.int32)
    rc = lib().orc_sourcetally(len(prt), prt.ctypes.data_as(C.c_void_p), _ptr(isvacant, ip), nx, ng,
                               _ptr(f64(grid.xarr), dp), _ptr(f64(groups.wl), dp), _ptr(en, dp), _ptr(num, ip))
    return rc, en, num   # (ng, nx) arrays = Fortran src_energy(ncell, ng)


# ---------------------------------------------------------------- sources
def make_source_particles(grid, groups, radtemp, L_bol, src_ns, npart=None, ioffset=0, rngmode=0, seed=0,
                          isvacant=None):
    """sourceenergy + sourcenumbers + vacancies + interior_source +
    source_transformdirection with the reference's mzran stream (rngmode 0)
    or the per-particle Philox streams of the GPU source kernel (rngmode 1)."""
    nx, ng = grid.nx, groups.ng
    emit = np.zeros(nx)
    tot = np.zeros(1)
    xarr = f64(grid.xarr)
    lib().orc_sourceenergy(nx, _ptr(xarr, dp), _ptr(f64(radtemp), dp), L_bol, _ptr(emit, dp), _ptr(tot, dp))
    npart = src_ns if npart is None else npart
    nvol = np.zeros(nx, dtype=np.int32)
    nnew = lib().orc_sourcenumbers(nx, _ptr(emit, dp), 1.0, src_ns, src_ns if isvacant is None else
                                   int(isvacant.sum()), _ptr(nvol, ip))
    if nnew < 0:
        raise RuntimeError(f"sourcenumbers failed: {nnew}")
    prt = np.zeros(npart, dtype=PACKET_DTYPE)
    isv = np.ones(npart, dtype=np.int32) if isvacant is None else isvacant.copy()
    st = rnd_init(1, ioffset)
    rc = lib().orc_interior_source(nx, ng, _ptr(xarr, dp), _ptr(f64(grid.vxarr), dp),
                                   _ptr(f64(groups.wlinv), dp), _ptr(f64(radtemp), dp), _ptr(emit, dp), 1.0,
                                   _ptr(nvol, ip), npart, prt.ctypes.data_as(C.c_void_p), _ptr(isv, ip),
                                   st.ctypes.data_as(C.c_void_p), rngmode, seed)
    if rc != 0:
        raise RuntimeError(f"interior_source failed: {rc}")
    return prt, isv, emit, nvol, float(tot[0])


# ---------------------------------------------------------------- equation of state
def partition(ion, temp):
    """ionsmod.f:206-215 at one temperature: q (nelem, nstage)."""
    ni = np.ascontiguousarray(ion.ni, dtype=np.int32)
    nl = np.ascontiguousarray(ion.nlevel, dtype=np.int32)
    g, e = f64(ion.glev), f64(ion.elev)
    q = np.zeros(ion.e.shape)
    lib().orc_partition(len(ni), ion.e.shape[1], g.shape[2], _ptr(ni, ip), _ptr(nl, ip), _ptr(g, dp), _ptr(e, dp),
                        float(temp), _ptr(q, dp))
    return q


def saha_eos(ion, q, temp, natom, vol, natomfr, nelec0, acc=1e-8, noc=4):
    """ions_solve_eos + eos_update for every cell.  Returns nelec, oc and ginv
    as numpy (nelem, noc, ncell), iconv."""
    ni = np.ascontiguousarray(ion.ni, dtype=np.int32)
    e, qq, g1 = f64(ion.e), f64(q), f64(ion.g1)
    st = OrcIon(len(ni), e.shape[1], ni.ctypes.data, e.ctypes.data, qq.ctypes.data, g1.ctypes.data)
    t, na, v, fr = f64(temp), f64(natom), f64(vol), f64(natomfr)
    nc = len(t)
    nel = f64(nelec0).copy()
    oc = np.zeros((len(ni), noc, nc))
    ginv = np.zeros((len(ni), noc, nc))
    it = np.zeros(nc, dtype=np.int32)
    rc = lib().orc_saha_eos(C.byref(st), nc, _ptr(t, dp), _ptr(na, dp), _ptr(v, dp), _ptr(fr, dp), float(acc),
                            _ptr(nel, dp), int(noc), _ptr(oc, dp), _ptr(ginv, dp), _ptr(it, ip))
    if rc != 0:
        raise RuntimeError(f"orc_saha_eos stopped at cell {-rc - 1}")
    return nel, oc, ginv, it
