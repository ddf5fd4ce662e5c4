"""The opacity build as a differentiable torch function (spectral fitting).

``DifferentiableOpacity(hot, ion, q_temp, elem_mass)`` prepares a HotPath
context (groups, one-model grid and atomic data already set) and
``opacity(temp, rho, massfr)`` returns ``(cap, sig, capgrey, capross,
opaclump)`` as CUDA tensors that carry gradients back to the shell
temperatures, densities and mass fractions.  Forward and reverse mode are
the library's kernels (slg_dev_opacity_grad_forward / _backward); torch only
holds the buffers and the autograd graph.

Layouts: temp, rho (ncell); massfr (ncell, nelem); cap (ncell, ng) (group
fastest, gas_cap's layout before sngl); sig, capgrey, capross (ncell);
opaclump (ncell, 11).
"""
from __future__ import annotations

import numpy as np
import torch

from .capi import ptr


def _dev64(t):
    return t.detach().to(dtype=torch.float64).contiguous()


class _OpacityFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, temp, rho, massfr, engine):
        T, R, X = _dev64(temp), _dev64(rho), _dev64(massfr)
        out = engine._forward(T, R, X)
        ctx.engine = engine
        ctx.save_for_backward(T, R, X, *out)
        return out[1:]

    @staticmethod
    def backward(ctx, gcap, gsig, ggrey, gross, gol):
        T, R, X, nelec, cap, sig, grey, ross, ol = ctx.saved_tensors
        gT, gR, gX = ctx.engine._backward(T, R, X, nelec, cap, sig, grey, ross, ol, gcap, gsig, ggrey, gross, gol)
        return gT, gR, gX, None


class DifferentiableOpacity:
    """Opacity build with a hand-written adjoint, behind torch.autograd."""

    def __init__(self, hot, ion, q_temp: float, elem_mass, acc: float = 1e-14, tauddmc: float = 5.0,
                 taulump: float = 10.0, nelec0: float = 1.0):
        self.hot = hot
        self.acc, self.tauddmc, self.taulump = float(acc), float(tauddmc), float(taulump)
        hot.set_ions(ion, q_temp)
        m = np.ascontiguousarray(elem_mass, dtype=np.float64)
        hot._check(hot.lib.slg_set_element_masses(hot.h, len(m), ptr(m)))
        self.nelem = len(m)
        self.device = torch.device("cuda", hot.device)
        self.nelec = torch.full((hot.nx,), float(nelec0), dtype=torch.float64, device=self.device)

    def opacity(self, temp, rho, massfr):
        return _OpacityFn.apply(temp, rho, massfr, self)

    def _sync(self):
        torch.cuda.ExternalStream(self.hot.stream(), device=self.device).synchronize()

    # ---------------------------------------------------------------- kernels
    def _forward(self, T, R, X):
        nc, ng = self.hot.nx, self.hot.ng
        e = lambda *s: torch.empty(s, dtype=torch.float64, device=self.device)
        torch.cuda.current_stream(self.device).synchronize()  # inputs come from torch's stream
        nelec = self.nelec.clone()
        cap, sig, grey, ross, ol = e(nc, ng), e(nc), e(nc), e(nc), e(nc, 11)
        self.hot._check(self.hot.lib.slg_dev_opacity_grad_forward(
            self.hot.h, ptr(T), ptr(R), ptr(X), self.acc, self.tauddmc, self.taulump, ptr(nelec), ptr(cap),
            ptr(sig), ptr(grey), ptr(ross), ptr(ol)))
        self._sync()
        self.nelec = nelec.clone()  # start value of the next solve, as the reference keeps gas_nelec
        return nelec, cap, sig, grey, ross, ol

    def _backward(self, T, R, X, nelec, cap, sig, grey, ross, ol, gcap, gsig, ggrey, gross, gol):
        c = lambda g: None if g is None else _dev64(g)
        gcap, gsig, ggrey, gross, gol = c(gcap), c(gsig), c(ggrey), c(gross), c(gol)
        gT, gR, gX = torch.empty_like(T), torch.empty_like(R), torch.empty_like(X)
        torch.cuda.current_stream(self.device).synchronize()  # gradients were produced on torch's stream
        self.hot._check(self.hot.lib.slg_dev_opacity_grad_backward(
            self.hot.h, ptr(T), ptr(R), ptr(X), self.acc, self.tauddmc, self.taulump, ptr(nelec), ptr(cap),
            ptr(sig), ptr(grey), ptr(ross), ptr(ol), ptr(gcap), ptr(gsig), ptr(ggrey), ptr(gross), ptr(gol),
            ptr(gT), ptr(gR), ptr(gX)))
        self._sync()
        return gT, gR, gX
