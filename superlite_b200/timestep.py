"""Device-resident driver of one SuperLite hot-path timestep.

Mirrors the order of the reference's iteration (superlite.f90:157-222):
physical_opacity -> opacity_planckmean/rossmean (gas_update.f:147-152) ->
leakage_opacity + emission_probability (superlite.f90:177-178) ->
sourcetally (:193) -> particle_advance (:202) -> fluxtally (:219).

All buffers are allocated once; one ``step()`` queues only libslg kernels on
the context's stream (plus one device-to-device restore of the source
particles, which stands in for the source generation that precedes the hot
path in the reference).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import capi
from .api import HotPath, PACKET_DTYPE
from .capi import ptr



class DeviceTimestep:
    def __init__(self, hot: HotPath, case, params, npart: int = 0, particles: np.ndarray = None,
                 isvacant: np.ndarray = None, flx_wl=None, precision=0):
        self.hot = hot
        self.params = params
        self.precision = precision
        dev = torch.device("cuda", hot.device)
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
        g = case.gas
        nc, ng = case.grid.nx, case.groups.ng
        self.nc, self.ng = nc, ng
        hot.set_groups(case.groups.wl)
        hot.set_grid(case.grid.xarr, case.grid.vxarr, case.grid.vol, case.grid.divv)
        hot.set_atomic_data(g.ion_ni, g.oc.shape[1], case.lines, case.bf_ph1, case.bf_ph2, case.ff_gff)
        self.gas = dict(temp=f64(g.temp), natom=f64(g.natom), nelec=f64(g.nelec), vol=f64(case.grid.vol),
                        mass=f64(g.mass), natomfr=f64(g.natomfr), oc=f64(g.oc), ginv=f64(g.ginv))
        self.tempinv = 1.0 / self.gas["temp"]
        self.sig = torch.empty(nc, dtype=torch.float64, device=dev)
        self.cap = torch.empty((nc, ng), dtype=torch.float32, device=dev)
        self.emiss = torch.empty((nc, ng), dtype=torch.float32, device=dev)
        self.capgrey = torch.empty(nc, dtype=torch.float64, device=dev)
        self.capross = torch.empty(nc, dtype=torch.float64, device=dev)
        self.opaclump = torch.empty((nc, 11), dtype=torch.float64, device=dev)
        self.emitprob = torch.empty((nc, hot.nep), dtype=torch.float64, device=dev)
        self.tally = torch.empty(nc, dtype=torch.float64, device=dev)
        self.jrad = torch.empty((nc, ng), dtype=torch.float64, device=dev)
        self.eamp = torch.empty(nc, dtype=torch.float64, device=dev)
        self.mswap = torch.empty(nc, dtype=torch.int32, device=dev)
        self.src_energy = torch.empty((ng, nc), dtype=torch.float64, device=dev)
        self.src_number = torch.empty((ng, nc), dtype=torch.int32, device=dev)
        fw = case.groups.wl if flx_wl is None else flx_wl
        self.flx_wl = f64(fw)
        self.flx_ng = len(fw) - 1
        self.lum = torch.empty(self.flx_ng, dtype=torch.float64, device=dev)
        self.lumdev = torch.empty_like(self.lum)
        self.lumnum = torch.empty(self.flx_ng, dtype=torch.int32, device=dev)
        if particles is not None:
            assert particles.dtype == PACKET_DTYPE
            raw = torch.as_tensor(particles.view(np.float64).reshape(-1, 8))
            self.prt0 = raw.to(dev)
            self.isv0 = torch.as_tensor(np.ascontiguousarray(isvacant, dtype=np.int32)).to(dev)
            npart = particles.shape[0]
        else:
            self.prt0 = self.isv0 = None  # particles are made on the device (interior_source)
        self.prt = torch.empty((npart, 8), dtype=torch.float64, device=dev)
        self.isv = torch.ones(npart, dtype=torch.int32, device=dev)
        self.npart = npart
        gp = capi.SlgGas(*[ptr(self.gas[k]) for k in ("temp", "natom", "nelec", "vol", "mass", "natomfr", "oc", "ginv")])
        self._gas = gp
        self._flags = capi.SlgOpacityFlags(0, 0, 0, 0, 1, 0.0)
        self._tin = HotPath.transport_in(self.tempinv, self.sig, self.capgrey, self.emitprob, self.opaclump, self.cap,
                                         params, precision)
        self._tout = capi.SlgTransportOut(ptr(self.tally), ptr(self.jrad), ptr(self.eamp), ptr(self.mswap), 0.0, 0.0, 0.0)
        self.stream = torch.cuda.ExternalStream(hot.stream(), device=dev)

    def _chk(self, rc):
        self.hot._check(rc)

    def opacity(self):
        L, h = self.hot.lib, self.hot.h
        self._chk(L.slg_dev_physical_opacity(h, C.byref(self._gas), C.byref(self._flags), ptr(self.sig), ptr(self.cap),
                                             ptr(self.emiss), None))
        self._chk(L.slg_dev_opacity_means(h, ptr(self.gas["temp"]), ptr(self.sig), ptr(self.cap), ptr(self.capgrey),
                                          ptr(self.capross)))

    def coefficients(self):
        L, h = self.hot.lib, self.hot.h
        p = self.params
        self._chk(L.slg_dev_leakage_opacity11(h, ptr(self.tempinv), ptr(self.sig), ptr(self.cap), None, p.tauddmc,
                                              p.taulump, ptr(self.opaclump)))
        self._chk(L.slg_dev_emission_probability(h, ptr(self.tempinv), ptr(self.cap), ptr(self.capgrey),
                                                 ptr(self.emitprob)))

    def restore_particles(self):
        if self.prt0 is None:
            return
        with torch.cuda.stream(self.stream):
            self.prt.copy_(self.prt0)
            self.isv.copy_(self.isv0)

    def transport(self, seed):
        L, h = self.hot.lib, self.hot.h
        self._chk(L.slg_dev_sourcetally(h, self.npart, ptr(self.prt), ptr(self.isv), ptr(self.src_energy),
                                        ptr(self.src_number)))
        self._tout.tot_evelo = self._tout.tot_eout = self._tout.tot_sflux = 0.0
        self._chk(L.slg_dev_particle_advance(h, C.byref(self._tin), ptr(self.prt), ptr(self.isv), self.npart, seed,
                                             C.byref(self._tout)))

    def autotune(self, seed=0, nsample=200_000):
        """Pick the fastest transport-kernel variant on a copy of the current
        particles (call after the particles are in place).  Returns (variant, ms)."""
        L, h = self.hot.lib, self.hot.h
        best = C.c_int32(0)
        ms = (C.c_float * 4)()
        self._chk(L.slg_autotune_transport(h, C.byref(self._tin), ptr(self.prt), ptr(self.isv), self.npart, seed,
                                           int(nsample), C.byref(best), ms))
        return int(best.value), [float(m) for m in ms]

    def fluxtally(self):
        L, h = self.hot.lib, self.hot.h
        self._chk(L.slg_dev_fluxtally(h, self.npart, ptr(self.prt), ptr(self.isv), self.flx_ng, ptr(self.flx_wl),
                                      ptr(self.lum), ptr(self.lumdev), ptr(self.lumnum)))

    def step(self, seed):
        """Queue one full timestep; call sync() to complete the transport counters."""
        self.restore_particles()
        self.opacity()
        self.coefficients()
        self.transport(seed)
        self.fluxtally()

    def sync(self):
        self.hot.sync()  # also folds the transport counters into self._tout
        return self.counters()

    def counters(self):
        from .api import transport_out_dict
        return transport_out_dict(self._tout)


class BatchTimestep:
    """One timestep of many independent models in one context (slg_set_models),
    device resident: analytic grey opacity, Planck/Rosseland
    means, leakage opacities, emission probabilities, source particles, the
    source tally, one persistent particle loop over every model's particles
    (precision 1) and per-model flux tallies.  ``capture(nsteps, seed)``
    records nsteps such steps in one CUDA graph; ``replay()`` runs it."""

    def __init__(self, hot: HotPath, batch, params, precision: int = 1, L_bol: float = 1e42):
        self.hot = hot
        self.params = params
        self.precision = precision
        b = batch
        hot.set_groups(b.groups.wl)
        hot.set_models(b.nx, b.npart, b.xarr, b.vxarr, b.vol, b.divv)
        dev = torch.device("cuda", hot.device)
        nc, ng = int(b.nx.sum()), b.groups.ng
        self.nc, self.ng, self.nmodel = nc, ng, len(b.nx)
        self.npart = int(b.npart.sum())
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
        e64 = lambda *s: torch.empty(s, dtype=torch.float64, device=dev)
        self.temp, self.rho = f64(b.temp), f64(b.rho)
        self.tempinv = 1.0 / self.temp
        self.sig, self.capgrey, self.capross = e64(nc), e64(nc), e64(nc)
        self.cap = torch.empty((nc, ng), dtype=torch.float32, device=dev)
        self.opaclump = e64(nc, 11)
        self.emitprob = e64(nc, hot.nep)
        self.tally, self.jrad, self.eamp = e64(nc), e64(nc, ng), e64(nc)
        self.mswap = torch.empty(nc, dtype=torch.int32, device=dev)
        self.src_energy = e64(ng, nc)
        self.src_number = torch.empty((ng, nc), dtype=torch.int32, device=dev)
        self.flx_wl = f64(b.groups.wl)
        self.lum, self.lumdev = e64(self.nmodel, ng), e64(self.nmodel, ng)
        self.lumnum = torch.empty((self.nmodel, ng), dtype=torch.int32, device=dev)
        self.prt = torch.empty((self.npart, 8), dtype=torch.float64, device=dev)
        self.isv = torch.ones(self.npart, dtype=torch.int32, device=dev)
        self.emit, _ = hot.sourceenergy(b.temp, L_bol)
        self.nvol, self.nnew = hot.models_sourcenumbers(self.emit, b.npart)
        self._tin = HotPath.transport_in(self.tempinv, self.sig, self.capgrey, self.emitprob, self.opaclump,
                                         self.cap, params, precision)
        self._tout = capi.SlgTransportOut(ptr(self.tally), ptr(self.jrad), ptr(self.eamp), ptr(self.mswap),
                                          0.0, 0.0, 0.0)
        self.stream = torch.cuda.ExternalStream(hot.stream(), device=dev)

    def _chk(self, rc):
        self.hot._check(rc)

    def step(self, seed: int):
        self.prepare(seed)
        self.finish(seed)

    def prepare(self, seed: int):
        """Sources, opacities and coefficients of a step (everything before the particle loop)."""
        L, h, p = self.hot.lib, self.hot.h, self.params
        self.hot.interior_source(self.temp, self.emit, self.nvol, self.prt, self.isv, seed=2 * seed)
        self._chk(L.slg_dev_analytic_opacity(h, ptr(self.temp), ptr(self.rho), 1, 1e18, -1.5, 2.0, 0.0, 0.0, 0.0,
                                             0.0, 0.0, ptr(self.sig), ptr(self.cap)))
        self._chk(L.slg_dev_opacity_means(h, ptr(self.temp), ptr(self.sig), ptr(self.cap), ptr(self.capgrey),
                                          ptr(self.capross)))
        self._chk(L.slg_dev_leakage_opacity11(h, ptr(self.tempinv), ptr(self.sig), ptr(self.cap), None, p.tauddmc,
                                              p.taulump, ptr(self.opaclump)))
        self._chk(L.slg_dev_emission_probability(h, ptr(self.tempinv), ptr(self.cap), ptr(self.capgrey),
                                                 ptr(self.emitprob)))
        self._chk(L.slg_dev_sourcetally(h, self.npart, ptr(self.prt), ptr(self.isv), ptr(self.src_energy),
                                        ptr(self.src_number)))

    def finish(self, seed: int):
        """The particle loop over every model and the per-model flux tallies."""
        self.transport(seed)
        self.flux()

    def transport(self, seed: int):
        """The particle loop over every model (precision as set at construction
        or by set_precision)."""
        L, h = self.hot.lib, self.hot.h
        self._tout.tot_evelo = self._tout.tot_eout = self._tout.tot_sflux = 0.0
        self._chk(L.slg_dev_particle_advance(h, C.byref(self._tin), ptr(self.prt), ptr(self.isv), self.npart,
                                             2 * seed + 1, C.byref(self._tout)))

    def set_precision(self, precision: int):
        """0: the FP64 particle loop (reference arithmetic) over all models in one
        launch; 1: the mixed-precision loop."""
        self.precision = precision
        self._tin.precision = int(precision)

    def flux(self):
        """fluxtally per model (also frees the escaped particles' slots)."""
        self._chk(self.hot.lib.slg_dev_fluxtally(self.hot.h, self.npart, ptr(self.prt), ptr(self.isv), self.ng,
                                                 ptr(self.flx_wl), ptr(self.lum), ptr(self.lumdev),
                                                 ptr(self.lumnum)))

    def autotune(self, seed=0, nsample=1_000_000):
        best = C.c_int32(0)
        ms = (C.c_float * 4)()
        self._chk(self.hot.lib.slg_autotune_transport(self.hot.h, C.byref(self._tin), ptr(self.prt), ptr(self.isv),
                                                      self.npart, seed, int(min(nsample, self.npart)),
                                                      C.byref(best), ms))
        return int(best.value), [float(m) for m in ms]

    def capture(self, nsteps: int, seed: int):
        self.hot.graph_begin()
        for k in range(nsteps):
            self.step(seed + k)
        self.hot.graph_end()

    def replay(self, n: int = 1):
        self.hot.graph_launch(n)

    def sync(self):
        self.hot.sync()
