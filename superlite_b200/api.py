"""Python host layer over libslg, mirroring the reference's hot-path routines.

Each method of :class:`HotPath` stands for one argument-less Fortran
subroutine of the reference and takes the module arrays it reads as numpy
arrays (host path, through the ``slg_*`` entry points) or torch CUDA tensors
(device path, through the ``slg_dev_*`` entry points):

=====================  ==============================================
method                 reference routine
=====================  ==============================================
physical_opacity       GAS/physical_opacity.f:3-357
analytic_opacity       GAS/analytic_opacity.f90:3-77
opacity_means          GAS/opacity_planckmean.f + GAS/opacity_rossmean.f
leakage_opacity        GRID/leakage_opacity11.f90:3-174
emission_probability   GRID/emission_probability.f90:3-67
particle_advance       particle_advance.f90:4-327 (+ transport11, diffusion11)
fluxtally              fluxtally.f:3-61
sourcetally            sourcetally.f:3-48
=====================  ==============================================

Errors: a nonzero status raises :class:`~superlite_b200.capi.SlgError`;
transport errors carry the reference's ierr codes (1, 3, 4, 17, 100, 102)
when ``errorfatal`` is set, as the reference stops on them
(particle_advance.f90:262-265).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import capi
from .capi import SlgError, ptr

PACKET_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("mu", "<f8"),
                         ("om", "<f8"), ("e", "<f8"), ("e0", "<f8"), ("wl", "<f8")])


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _is_torch(a):
    return hasattr(a, "data_ptr") and not isinstance(a, np.ndarray)


class HotPath:
    """One libslg context (one device, one stream)."""

    def __init__(self, device: int = 0):
        self.lib = capi.load()
        h = self.lib.slg_create(device)
        if not h:
            raise SlgError(-1, f"slg_create({device}) failed: no usable CUDA device")
        self.h = h
        self.device = device
        self.ng = self.nx = 0
        self._keep = []

    def close(self):
        if getattr(self, "h", None):
            self.lib.slg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise SlgError(rc, self.lib.slg_last_error(self.h).decode())
        return rc

    @property
    def nep(self):
        return int(round(np.sqrt(float(self.ng))))

    @property
    def nepg(self):
        return int(np.ceil(self.ng / (self.nep + 1.0)))

    def stream(self):
        return self.lib.slg_stream(self.h)

    def sync(self):
        self._check(self.lib.slg_sync(self.h))

    # ------------------------------------------------------------- set-up
    def set_groups(self, grp_wl):
        wl = _f64(grp_wl)
        self._check(self.lib.slg_set_groups(self.h, len(wl) - 1, ptr(wl)))
        self.ng = len(wl) - 1
        self.grp_wl = wl

    def set_grid(self, xarr, vxarr, vol, divv):
        x, vx, v, dv = _f64(xarr), _f64(vxarr), _f64(vol), _f64(divv)
        self._check(self.lib.slg_set_grid(self.h, len(x) - 1, ptr(x), ptr(vx), ptr(v), ptr(dv)))
        self.nx = len(x) - 1
        self.xarr = x
        self.nmodel = 1

    def set_models(self, nx, npart, xarr, vxarr, vol, divv):
        """Several independent models in this context (slg_set_models): nx[m]
        shells and npart[m] particle slots each; xarr/vxarr concatenate each
        model's nx[m]+1 edges, vol/divv each model's cells."""
        n = np.ascontiguousarray(nx, dtype=np.int32)
        npt = np.ascontiguousarray(npart, dtype=np.int64)
        x, vx, v, dv = _f64(xarr), _f64(vxarr), _f64(vol), _f64(divv)
        assert len(x) == n.sum() + len(n) and len(v) == n.sum() and len(npt) == len(n)
        self._check(self.lib.slg_set_models(self.h, len(n), ptr(n), ptr(npt), ptr(x), ptr(vx), ptr(v), ptr(dv)))
        self.nx = int(n.sum())
        self.xarr = x
        self.nmodel = len(n)
        self.model_nx = n
        self.model_npart = npt

    def set_atomic_data(self, ion_ni, nstage, lines, bf_ph1, bf_ph2, ff_gff):
        ni = np.ascontiguousarray(ion_ni, dtype=np.int32)
        ln = np.ascontiguousarray(lines)
        p1, p2, g = _f32(bf_ph1), _f32(bf_ph2), _f64(ff_gff)
        self._check(self.lib.slg_set_atomic_data(self.h, len(ni), int(nstage), ptr(ni), len(ln), ptr(ln),
                                                 ptr(p1), ptr(p2), ptr(g)))

    # ------------------------------------------------------------- opacity
    def physical_opacity(self, temp, natom, nelec, vol, mass, natomfr, oc, ginv, ngs=1, nobb=False,
                         nobf=False, noff=False, nothmson=False, opacmixrossel=0.0, want_cap64=False):
        """Host path.  Returns dict(sig, cap (ncell,ng) f32, emiss, cap64, sanity)."""
        nc, ng = self.nx, self.ng
        arrs = [_f64(a) for a in (temp, natom, nelec, vol, mass, natomfr, oc, ginv)]
        gas = capi.SlgGas(*[ptr(a) for a in arrs])
        fl = capi.SlgOpacityFlags(int(nobb), int(nobf), int(noff), int(nothmson), int(ngs), float(opacmixrossel))
        sig = np.zeros(nc)
        cap = np.zeros((nc, ng), dtype=np.float32)
        emiss = np.zeros((nc, ng), dtype=np.float32)
        cap64 = np.zeros((ng, nc)) if want_cap64 else None
        san = np.zeros(1, dtype=np.int32)
        self._check(self.lib.slg_physical_opacity(self.h, C.byref(gas), C.byref(fl), ptr(sig), ptr(cap), ptr(emiss),
                                                  ptr(cap64), ptr(san)))
        return dict(sig=sig, cap=cap, emiss=emiss, cap64=None if cap64 is None else np.ascontiguousarray(cap64.T),
                    sanity=int(san[0]))

    def physical_opacity_dev(self, gas_t: dict, out: dict, ngs=1, nobb=False, nobf=False, noff=False,
                             nothmson=False, opacmixrossel=0.0):
        """Device path: gas_t holds torch CUDA tensors; out holds sig, cap, emiss (and optional cap64)."""
        keys = ("temp", "natom", "nelec", "vol", "mass", "natomfr", "oc", "ginv")
        gas = capi.SlgGas(*[ptr(gas_t[k]) for k in keys])
        fl = capi.SlgOpacityFlags(int(nobb), int(nobf), int(noff), int(nothmson), int(ngs), float(opacmixrossel))
        self._check(self.lib.slg_dev_physical_opacity(self.h, C.byref(gas), C.byref(fl), ptr(out["sig"]),
                                                      ptr(out["cap"]), ptr(out["emiss"]), ptr(out.get("cap64"))))

    def analytic_opacity(self, temp, rho, kind=1, capcoef=1e18, captpwr=-1.5, caprpwr=2.0, sigcoef=0.0,
                         sigtpwr=0.0, sigrpwr=0.0, ldisp1=1.0, ldisp2=1.0):
        t, r = _f64(temp), _f64(rho)
        sig = np.zeros(self.nx)
        cap = np.zeros((self.nx, self.ng), dtype=np.float32)
        self._check(self.lib.slg_analytic_opacity(self.h, ptr(t), ptr(r), int(kind), capcoef, captpwr, caprpwr,
                                                  sigcoef, sigtpwr, sigrpwr, ldisp1, ldisp2, ptr(sig), ptr(cap)))
        return sig, cap

    def opacity_means(self, temp, sig, cap):
        if _is_torch(cap):
            import torch
            grey = torch.empty(self.nx, dtype=torch.float64, device=cap.device)
            ross = torch.empty_like(grey)
            self._check(self.lib.slg_dev_opacity_means(self.h, ptr(temp), ptr(sig), ptr(cap), ptr(grey), ptr(ross)))
            return grey, ross
        t, s, c = _f64(temp), _f64(sig), _f32(cap)
        grey, ross = np.zeros(self.nx), np.zeros(self.nx)
        self._check(self.lib.slg_opacity_means(self.h, ptr(t), ptr(s), ptr(c), ptr(grey), ptr(ross)))
        return grey, ross

    # ------------------------------------------------------------- grid coefficients
    def leakage_opacity(self, tempinv, sig, cap, capemit=None, tauddmc=5.0, taulump=10.0):
        if _is_torch(cap):
            import torch
            ol = torch.empty((self.nx, 11), dtype=torch.float64, device=cap.device)
            self._check(self.lib.slg_dev_leakage_opacity11(self.h, ptr(tempinv), ptr(sig), ptr(cap), ptr(capemit),
                                                           tauddmc, taulump, ptr(ol)))
            return ol
        t, s, c = _f64(tempinv), _f64(sig), _f32(cap)
        ce = None if capemit is None else _f32(capemit)
        ol = np.zeros((self.nx, 11))
        self._check(self.lib.slg_leakage_opacity11(self.h, ptr(t), ptr(s), ptr(c), ptr(ce), tauddmc, taulump, ptr(ol)))
        return ol

    def emission_probability(self, tempinv, cap, capgrey):
        if _is_torch(cap):
            import torch
            ep = torch.empty((self.nx, self.nep), dtype=torch.float64, device=cap.device)
            self._check(self.lib.slg_dev_emission_probability(self.h, ptr(tempinv), ptr(cap), ptr(capgrey), ptr(ep)))
            return ep
        t, c, g = _f64(tempinv), _f32(cap), _f64(capgrey)
        ep = np.zeros((self.nx, self.nep))
        self._check(self.lib.slg_emission_probability(self.h, ptr(t), ptr(c), ptr(g), ptr(ep)))
        return ep

    # ------------------------------------------------------------- transport
    @staticmethod
    def transport_in(tempinv, sig, capgrey, emitprob, opaclump, cap, params, precision=0):
        tin = capi.SlgTransportIn(ptr(tempinv), ptr(sig), ptr(capgrey), ptr(emitprob), ptr(opaclump), ptr(cap),
                                  float(params.tauddmc), float(params.taulump), int(params.puretran),
                                  int(params.noampfact), int(params.errorfatal), int(params.thm_aniso),
                                  int(params.dogrdtally), int(precision), int(params.max_steps))
        return tin

    def particle_advance(self, tables: dict, prt, isvacant, params, seed=0, precision=0, trace=False,
                         totals=(0.0, 0.0, 0.0)):
        """Host path (numpy).  tables: tempinv, sig, capgrey, emitprob, opaclump, cap.
        prt (PACKET_DTYPE) and isvacant (int32) are updated in place."""
        keep = dict(tempinv=_f64(tables["tempinv"]), sig=_f64(tables["sig"]), capgrey=_f64(tables["capgrey"]),
                    emitprob=_f64(tables["emitprob"]), opaclump=_f64(tables["opaclump"]), cap=_f32(tables["cap"]))
        assert prt.dtype == PACKET_DTYPE and prt.flags.c_contiguous
        assert isvacant.dtype == np.int32 and isvacant.flags.c_contiguous
        tin = self.transport_in(**keep, params=params, precision=precision)
        nx, ng = self.nx, self.ng
        tally, jrad, eamp = np.zeros(nx), np.zeros((nx, ng)), np.zeros(nx)
        mswap = np.zeros(nx, dtype=np.int32)
        out = capi.SlgTransportOut(ptr(tally), ptr(jrad), ptr(eamp), ptr(mswap), *totals)
        th = tn = None
        if trace:
            th = np.zeros(len(prt), dtype=np.uint64)
            tn = np.zeros(len(prt), dtype=np.int32)
            self._check(self.lib.slg_set_trace(self.h, ptr(th), ptr(tn)))
        try:
            rc = self.lib.slg_particle_advance(self.h, C.byref(tin), ptr(prt), ptr(isvacant), len(prt), seed,
                                               C.byref(out))
        finally:
            if trace:
                self.lib.slg_set_trace(self.h, None, None)
        if rc < 0:
            self._check(rc)
        res = _out_dict(out)
        res.update(rc=rc, tally=tally, jrad=jrad, eamp=eamp, methodswap=mswap)
        if trace:
            res["trace_hash"], res["trace_nstep"] = th, tn
        return res

    def particle_advance_dev(self, tables: dict, prt, isvacant, tally, jrad, eamp, params, seed=0, precision=0,
                             methodswap=None):
        """Device path: every array is a torch CUDA tensor; returns the SlgTransportOut (valid after sync())."""
        tin = self.transport_in(tables["tempinv"], tables["sig"], tables["capgrey"], tables["emitprob"],
                                tables["opaclump"], tables["cap"], params, precision)
        out = capi.SlgTransportOut(ptr(tally), ptr(jrad), ptr(eamp), ptr(methodswap), 0.0, 0.0, 0.0)
        self._keep = [tin, out]
        self._check(self.lib.slg_dev_particle_advance(self.h, C.byref(tin), ptr(prt), ptr(isvacant), int(prt.shape[0]),
                                                      seed, C.byref(out)))
        return out

    def autotune_transport(self, tables: dict, prt, isvacant, params, precision=0, seed=0, nsample=1_000_000):
        """slg_autotune_transport on device tensors (torch CUDA): times every
        variant of the particle loop of `precision` on a copy of the first
        nsample particles and keeps the fastest for this context.  Returns
        (variant, [ms per variant])."""
        tin = self.transport_in(tables["tempinv"], tables["sig"], tables["capgrey"], tables["emitprob"],
                                tables["opaclump"], tables["cap"], params, precision)
        best = C.c_int32(0)
        ms = (C.c_float * 4)()
        npart = int(prt.shape[0])
        self._check(self.lib.slg_autotune_transport(self.h, C.byref(tin), ptr(prt), ptr(isvacant), npart, int(seed),
                                                    int(min(nsample, npart)), C.byref(best), ms))
        return int(best.value), [float(m) for m in ms]

    def fluxtally(self, prt, isvacant, flx_wl):
        rows = getattr(self, "nmodel", 1)  # one row of groups per model
        if _is_torch(prt):
            import torch
            ng = flx_wl.shape[0] - 1
            shape = (rows, ng) if rows > 1 else (ng,)
            lum = torch.empty(shape, dtype=torch.float64, device=prt.device)
            dev = torch.empty_like(lum)
            num = torch.empty(shape, dtype=torch.int32, device=prt.device)
            self._check(self.lib.slg_dev_fluxtally(self.h, int(prt.shape[0]), ptr(prt), ptr(isvacant), ng, ptr(flx_wl),
                                                   ptr(lum), ptr(dev), ptr(num)))
            return lum, dev, num
        w = _f64(flx_wl)
        ng = len(w) - 1
        shape = (rows, ng) if rows > 1 else (ng,)
        lum, dev, num = np.zeros(shape), np.zeros(shape), np.zeros(shape, dtype=np.int32)
        self._check(self.lib.slg_fluxtally(self.h, len(prt), ptr(prt), ptr(isvacant), ng, ptr(w), ptr(lum), ptr(dev),
                                           ptr(num)))
        return lum, dev, num

    # ------------------------------------------------------------- sources
    def sourceenergy(self, radtemp, L_bol):
        """SOURCE/sourceenergy.f90: grd_emit (ncell) and tot_sthermal."""
        t = _f64(radtemp)
        emit = np.zeros(self.nx)
        tot = np.zeros(1)
        self._check(self.lib.slg_sourceenergy(self.h, ptr(t), float(L_bol), ptr(emit), ptr(tot)))
        return emit, float(tot[0])

    def sourcenumbers(self, emit, src_ns, nvacant=None, srcepwr=1.0):
        """SOURCE/sourcenumbers.f90 (one rank): grd_nvol and src_nnew."""
        e = _f64(emit)
        nvol = np.zeros(self.nx, dtype=np.int32)
        n = self.lib.slg_sourcenumbers(self.h, ptr(e), float(srcepwr), int(src_ns),
                                       int(src_ns if nvacant is None else nvacant), ptr(nvol))
        if n < 0:
            self._check(int(n))
        return nvol, int(n)

    def models_sourcenumbers(self, emit, src_ns, nvacant=None, srcepwr=1.0):
        """sourcenumbers per model (slg_models_sourcenumbers)."""
        e = _f64(emit)
        ns = np.ascontiguousarray(src_ns, dtype=np.int64)
        nv = ns if nvacant is None else np.ascontiguousarray(nvacant, dtype=np.int64)
        nvol = np.zeros(self.nx, dtype=np.int32)
        n = self.lib.slg_models_sourcenumbers(self.h, ptr(e), float(srcepwr), ptr(ns), ptr(nv), ptr(nvol))
        if n < 0:
            self._check(int(n))
        return nvol, int(n)

    # ------------------------------------------------------------- equation of state
    def set_ions(self, ion, q_temp: float):
        """Ion data (workloads.IonTable) with the partition functions frozen at
        q_temp, as ions_solve_eos evaluates them once (ionsmod.f:206-215)."""
        ni = np.ascontiguousarray(ion.ni, dtype=np.int32)
        nl = np.ascontiguousarray(ion.nlevel, dtype=np.int32)
        g, el = _f64(ion.glev), _f64(ion.elev)
        q = np.zeros(ion.e.shape)
        self.lib.slg_partition_functions(len(ni), ion.e.shape[1], g.shape[2], ptr(ni), ptr(nl), ptr(g), ptr(el),
                                         float(q_temp), ptr(q))
        e, g1 = _f64(ion.e), _f64(ion.g1)
        self._check(self.lib.slg_set_ions(self.h, len(ni), e.shape[1], ptr(ni), ptr(e), ptr(q), ptr(g1)))
        self.ion_nelem = len(ni)
        return q

    def saha_eos(self, temp, natom, vol, natomfr, nelec0, acc=1e-8, noc=4):
        """ions_solve_eos + eos_update: returns nelec, oc, ginv ((nelem, noc, ncell)
        numpy, or torch tensors on the device when the inputs are) and iconv."""
        if _is_torch(temp):
            import torch
            dev = temp.device
            nel = nelec0.clone()
            oc = torch.empty((self.ion_nelem, noc, self.nx), dtype=torch.float64, device=dev)
            ginv = torch.empty_like(oc)
            it = torch.empty(self.nx, dtype=torch.int32, device=dev)
            self._check(self.lib.slg_dev_saha_eos(self.h, ptr(temp), ptr(natom), ptr(vol), ptr(natomfr), float(acc),
                                                  ptr(nel), int(noc), ptr(oc), ptr(ginv), ptr(it)))
            return nel, oc, ginv, it
        t, na, v, fr = _f64(temp), _f64(natom), _f64(vol), _f64(natomfr)
        nel = _f64(nelec0).copy()
        oc = np.zeros((self.ion_nelem, noc, self.nx))
        ginv = np.zeros_like(oc)
        it = np.zeros(self.nx, dtype=np.int32)
        self._check(self.lib.slg_saha_eos(self.h, ptr(t), ptr(na), ptr(v), ptr(fr), float(acc), ptr(nel), int(noc),
                                          ptr(oc), ptr(ginv), ptr(it)))
        return nel, oc, ginv, it

    # ------------------------------------------------------------- CUDA graphs
    def graph_begin(self):
        self._check(self.lib.slg_graph_begin(self.h))

    def graph_end(self):
        self._check(self.lib.slg_graph_end(self.h))

    def graph_launch(self, n=1):
        self._check(self.lib.slg_graph_launch(self.h, int(n)))

    def transport_totals(self, reset=False):
        """Counters summed over every particle_advance since the last reset."""
        out = capi.SlgTransportOut()
        rc = self.lib.slg_transport_totals(self.h, C.byref(out), 1 if reset else 0)
        if rc < 0:
            self._check(rc)
        return transport_out_dict(out)

    def interior_source(self, radtemp, emit, nvol, prt, isvacant, seed=0):
        """vacancies + interior_source + source_transformdirection.  numpy arrays are
        updated in place (host path); torch CUDA tensors use the device path."""
        e = _f64(emit)
        nv = np.ascontiguousarray(nvol, dtype=np.int32)
        nnew = C.c_int64(0)
        if _is_torch(prt):
            self._check(self.lib.slg_dev_interior_source(self.h, ptr(radtemp), ptr(e), ptr(nv), ptr(prt),
                                                         ptr(isvacant), int(prt.shape[0]), seed, C.byref(nnew)))
            return int(nnew.value)
        t = _f64(radtemp)
        self._check(self.lib.slg_interior_source(self.h, ptr(t), ptr(e), ptr(nv), ptr(prt), ptr(isvacant), len(prt),
                                                 seed, C.byref(nnew)))
        return int(nnew.value)

    def sourcetally(self, prt, isvacant):
        """Returns src_energy, src_number as (ng, ncell) arrays (Fortran (ncell, ng))."""
        if _is_torch(prt):
            import torch
            en = torch.empty((self.ng, self.nx), dtype=torch.float64, device=prt.device)
            num = torch.empty((self.ng, self.nx), dtype=torch.int32, device=prt.device)
            self._check(self.lib.slg_dev_sourcetally(self.h, int(prt.shape[0]), ptr(prt), ptr(isvacant), ptr(en),
                                                     ptr(num)))
            return en, num
        en = np.zeros((self.ng, self.nx))
        num = np.zeros((self.ng, self.nx), dtype=np.int32)
        self._check(self.lib.slg_sourcetally(self.h, len(prt), ptr(prt), ptr(isvacant), ptr(en), ptr(num)))
        return en, num


def _out_dict(out):
    return dict(tot_evelo=out.tot_evelo, tot_eout=out.tot_eout, tot_sflux=out.tot_sflux, npckt=out.npckt,
                nflux=out.nflux, nstepimc=out.nstepimc, nstepddmc=out.nstepddmc, nmethodswap=out.nmethodswap,
                nstepmax=out.nstepmax, ndist=np.array(list(out.ndist)), nposwarn=out.nposwarn, ierr=out.ierr,
                ierr_part=out.ierr_part)


def transport_out_dict(out):
    return _out_dict(out)
