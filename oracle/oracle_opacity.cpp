// oracle_opacity.cpp -- physical LTE opacity, analytic opacity and the Planck /
// Rosseland means of the reference, restated on the CPU.
// TEST INFRASTRUCTURE ONLY (parity checker for the CUDA product).
//
// GAS/physical_opacity.f:3-357, bfxsmod.f:65-153, GAS/analytic_opacity.f90:3-77,
// GAS/opacity_planckmean.f:3-27, GAS/opacity_rossmean.f:3-23.
// Single-threaded: the reference's OpenMP bb loop accumulates into a shared
// cap(i,igs) without atomics (physical_opacity.f:104-152) and is only exact
// with one thread.
#include <cfloat>
#include <cstring>
#include "oracle_internal.h"

using namespace orc;

namespace {
// bfxsmod.f:8-12
const int ll[7] = {0, 0, 1, 0, 1, 2, 0};
const int ninn[30] = {0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 3, 3, 3, 3, 3,
                      3, 3, 3, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5};
const int ntot[30] = {1, 1, 2, 2, 3, 3, 3, 3, 3, 3, 4, 4, 5, 5, 5,
                      5, 5, 5, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 7, 7};
// bf_ph1(6,7,30,30): (k, is, nz, ne) column-major
inline float PH1(const float* t, int k, int is, int nz, int ne) {
  return t[(k - 1) + 6 * ((is - 1) + 7 * ((nz - 1) + 30 * (ne - 1)))];
}
// bf_ph2(7,30,30): (k, nz, ne)
inline float PH2(const float* t, int k, int nz, int ne) {
  return t[(k - 1) + 7 * ((nz - 1) + 30 * (ne - 1))];
}
inline float sqf(float x) { return x * x; }  // real*4 ** 2, evaluated in single precision
}  // namespace

extern "C" {

// bfxsmod.f:65-153 (Verner et al. 1996 / Verner & Yakovlev 1995 fits).
double orc_bfxs(const float* ph1, const float* ph2, int nz, int ne, double e) {
  double xs = 0.0;
  if (nz < 1 || nz > 30) return xs;
  if (ne < 1 || ne > nz) return xs;
  int nout = ntot[ne - 1];
  if (nz > 18) {
    if (nz == ne) nout = 7;
    if (nz == ne + 1) {
      if (nz == 20 || nz == 21 || nz == 22 || nz == 25 || nz == 26) nout = 7;
    }
  }
  if (e < (double)PH1(ph1, 1, nout, nz, ne)) return xs;
  int nint_ = ninn[ne - 1];
  double einn;
  if (nz == 15 || nz == 17 || nz == 19 || (nz > 20 && nz != 26)) {
    einn = 0.0;
  } else {
    if (ne < 3) einn = (double)1.0e30f;
    else einn = (double)PH1(ph1, 1, nint_, nz, ne);
  }
  xs = 0.0;
  for (int is = 1; is <= nout; ++is) {
    if (e < (double)PH1(ph1, 1, is, nz, ne)) continue;
    if (is < nout && is > nint_ && e < einn) continue;
    if (is <= nint_ || e >= einn) {
      double p1 = -(double)PH1(ph1, 5, is, nz, ne);
      double y = e / (double)PH1(ph1, 2, is, nz, ne);
      double q = -0.5 * p1 - (double)ll[is - 1] - 5.5;
      double a = (double)PH1(ph1, 3, is, nz, ne) *
                 (sq(y - 1.0) + (double)sqf(PH1(ph1, 6, is, nz, ne)));
      double b = std::sqrt(y / (double)PH1(ph1, 4, is, nz, ne)) + 1.0;
      xs = xs + a * std::pow(y, q) * std::pow(b, p1);
    } else {
      double p1 = -(double)PH2(ph2, 4, nz, ne);
      double q = -0.5 * p1 - 5.5;
      double x = e / (double)PH2(ph2, 1, nz, ne) - (double)PH2(ph2, 6, nz, ne);
      double z = std::sqrt(x * x + (double)sqf(PH2(ph2, 7, nz, ne)));
      double a = (double)PH2(ph2, 2, nz, ne) * (sq(x - 1.0) + (double)sqf(PH2(ph2, 5, nz, ne)));
      double b = 1.0 + std::sqrt(z / (double)PH2(ph2, 3, nz, ne));
      xs = xs + a * std::pow(z, q) * std::pow(b, p1);
    }
  }
  return xs;
}

// GAS/physical_opacity.f:3-357
int orc_physical_opacity(const orc_opac_in* in, double* gas_sig, float* gas_cap,
                         float* gas_emiss, double* cap64) {
  const int nc = in->ncell, ng = in->ng, ngs = in->ngs, nelem = in->nelem, nst = in->nstage;
  const int ngsub = ng * ngs;
  auto CAP = [&](std::vector<double>& c, int i, int igs) -> double& {
    return c[(size_t)(i - 1) + (size_t)nc * (igs - 1)];
  };
  std::vector<double> cap((size_t)nc * ngsub, 0.0);
  // subgridded wavelength :65-78
  std::vector<double> wlsub(ngsub + 1);
  if (ngs == 1) {
    for (int k = 0; k <= ng; ++k) wlsub[k] = in->grp_wl[k];
  } else {
    int igs = 1;
    wlsub[0] = in->grp_wl[0];
    double help = 1.0 / ngs;
    for (int ig = 1; ig <= ng; ++ig)
      for (int i = 1; i <= ngs; ++i) {
        igs = igs + 1;
        wlsub[igs - 1] = (1.0 - i * help) * in->grp_wl[ig - 1] + i * help * in->grp_wl[ig];
      }
  }
  auto WLSUB = [&](int k) { return wlsub[k - 1]; };
  auto mass = [&](int i) { return in->mass[i - 1]; };
  // :81
  std::vector<double> hckt(nc);
  for (int i = 1; i <= nc; ++i) hckt[i - 1] = pc_hc / (pc_kb * in->temp[i - 1]);
  // :84-89
  for (int i = 1; i <= nc; ++i) {
    if (in->nothmson) gas_sig[i - 1] = 0.0;
    else {
      gas_sig[i - 1] = cthomson * in->nelec[i - 1] * in->natom[i - 1] / in->vol[i - 1];
      if (mass(i) <= 0.0) gas_sig[i - 1] = 0.0;
    }
  }
  auto ionlim = [&](int iz) {
    int m = in->ion_ni[iz - 1] - 1;
    return iz < m ? iz : m;
  };
  auto IDX = [&](int i, int ii, int iz) {
    return (size_t)(i - 1) + (size_t)nc * ((ii - 1) + (size_t)nst * (iz - 1));
  };
  // bound-bound :94-158
  if (!in->nobb) {
    std::vector<double> grndlev((size_t)nc * nst * nelem, 0.0);
    for (int iz = 1; iz <= nelem; ++iz)
      for (int i = 1; i <= nc; ++i) {
        if (mass(i) <= 0.0) continue;
        for (int ii = 1; ii <= ionlim(iz); ++ii)
          grndlev[IDX(i, ii, iz)] = in->oc[IDX(i, ii, iz)] * in->ginv[IDX(i, ii, iz)];
      }
    int iigs = 0;
    bool dirty = true;
    double phi = 0.0;
    std::vector<double> expfac(nc, 0.0);
    for (int64_t il = 0; il < in->nline; ++il) {
      const orc_bbxs& L = in->bb[il];
      double wl0 = (double)L.wl0 * pc_ang;
      int iz = L.iz, ii = L.ii;
      int igs;
      for (igs = iigs; igs <= ngsub; ++igs) {
        if (WLSUB(igs + 1) > wl0) break;
        dirty = true;
      }
      iigs = igs;
      if (igs < 1) continue;
      if (igs > ngsub) continue;
      if (dirty) {
        dirty = false;
        double wl = 0.5 * (WLSUB(igs) + WLSUB(igs + 1));
        double wlinv = 1.0 / wl;
        double dwl = WLSUB(igs + 1) - WLSUB(igs);
        for (int i = 0; i < nc; ++i) expfac[i] = 1.0 - std::exp(-(hckt[i] * wlinv));
        phi = wl * wl / (dwl * pc_c);
      }
      for (int i = 1; i <= nc; ++i) {
        if (mass(i) <= 0.0) continue;
        double ocggrnd = grndlev[IDX(i, ii, iz)];
        if (ocggrnd <= 0.0) continue;
        double caphelp = phi * (double)L.gxs * ocggrnd *
                         std::exp(-((double)L.chilw * hckt[i - 1])) * expfac[i - 1];
        CAP(cap, i, igs) = CAP(cap, i, igs) + caphelp;
      }
    }
  }
  // bound-free :163-195
  if (!in->nobf) {
    for (int igs = 1; igs <= ngsub; ++igs) {
      double wl = WLSUB(igs);
      double en = pc_hc / (pc_ev * wl);
      for (int iz = 1; iz <= nelem; ++iz)
        for (int ii = 1; ii <= ionlim(iz); ++ii) {
          int ie = iz - ii + 1;
          double xs = orc_bfxs(in->bf_ph1, in->bf_ph2, iz, ie, en);
          if (xs == 0.0) continue;
          for (int i = 1; i <= nc; ++i) {
            if (mass(i) <= 0.0) continue;
            CAP(cap, i, igs) = CAP(cap, i, igs) + xs * pc_mbarn * in->oc[IDX(i, ii, iz)];
          }
        }
    }
  }
  // free-free :200-247
  if (!in->noff) {
    const double c1 = ff_c1();
    const int ff_nu = 81, ff_ngg = 41;
    auto GFF = [&](int iu, int igg) { return in->ff_gff[(iu - 1) + ff_nu * (igg - 1)]; };
    std::vector<double> hlparr(nc);
    for (int i = 0; i < nc; ++i)
      hlparr[i] = sq(in->natom[i] / in->vol[i]) * in->nelec[i];
    for (int igs = 1; igs <= ngsub; ++igs) {
      double wl = WLSUB(igs);
      double wlinv = 1.0 / wl;
      for (int i = 1; i <= nc; ++i) {
        if (mass(i) <= 0.0) continue;
        double u = hckt[i - 1] * wlinv;
        double ru = 10.0 * (std::log10(u) + 4.0) + 1.0;
        int iu = ru < 1.0 ? 1 : (ru >= (double)(ff_nu - 1) ? ff_nu - 1 : (int)std::floor(ru));
        double du = ru - iu;
        double help = c1 * std::sqrt(hckt[i - 1]) * (1.0 - std::exp(-u)) * cube(wl) * hlparr[i - 1];
        for (int iz = 1; iz <= nelem; ++iz) {
          double gg = (double)(iz * iz) * pc_rydberg * hckt[i - 1];
          double rgg = 5.0 * (std::log10(gg) + 4.0) + 1.0;
          int igg = rgg < 1.0 ? 1 : (rgg >= (double)(ff_ngg - 1) ? ff_ngg - 1 : (int)std::floor(rgg));
          double dgg = rgg - igg;
          double gff = (1.0 - du) * (1.0 - dgg) * GFF(iu, igg) + du * (1.0 - dgg) * GFF(iu + 1, igg) +
                       (1.0 - du) * dgg * GFF(iu, igg + 1) + du * dgg * GFF(iu + 1, igg + 1);
          if (rgg > ff_ngg) gff = gff > 1.0 ? gff : 1.0;
          CAP(cap, i, igs) = CAP(cap, i, igs) +
                             help * gff * (double)(iz * iz) * in->natomfr[iz + (nelem + 1) * (i - 1)];
        }
      }
    }
  }
  // collapse subgridding :252-264
  if (ngs != 1) {
    double help = 1.0 / ngs;
    std::vector<double> capp(nc), capr(nc);
    for (int ig = 1; ig <= ng; ++ig) {
      int i0 = (ig - 1) * ngs + 1, j0 = i0 + ngs - 1;
      for (int c = 1; c <= nc; ++c) {
        double sp = 0.0, sr = 0.0;
        for (int k = i0; k <= j0; ++k) {
          double v = CAP(cap, c, k);
          if (v > 0.0) { sp = sp + v; sr = sr + 1.0 / v; }
        }
        capp[c - 1] = sp * help;
        capr[c - 1] = sr * help;
        if (capr[c - 1] > 0.0) capr[c - 1] = 1.0 / capr[c - 1];
      }
      for (int c = 1; c <= nc; ++c)
        CAP(cap, c, ig) = (1.0 - in->opacmixrossel) * capp[c - 1] + in->opacmixrossel * capr[c - 1];
    }
  }
  // save :267-279
  for (int i = 1; i <= nc; ++i)
    for (int ig = 1; ig <= ng; ++ig) {
      double v = CAP(cap, i, ig);
      gas_cap[(size_t)(ig - 1) + (size_t)ng * (i - 1)] = (float)v;
      if (cap64) cap64[(size_t)(i - 1) + (size_t)nc * (ig - 1)] = v;
      double em = 0.0;
      if (mass(i) > 0.0) {
        double wl = 0.5 * (in->grp_wl[ig] + in->grp_wl[ig - 1]);
        double B_nu = (wl * wl / pc_c) * orc_planck(wl, in->temp[i - 1]);
        em = 0.0 + v * B_nu;
      }
      gas_emiss[(size_t)(ig - 1) + (size_t)ng * (i - 1)] = (float)em;
    }
  // sanity check :282-291
  int j = 0;
  for (int i = 1; i <= nc; ++i) {
    if (mass(i) <= 0.0) continue;
    for (int ig = 1; ig <= ng; ++ig) {
      float v = gas_cap[(size_t)(ig - 1) + (size_t)ng * (i - 1)];
      if (v == 0.f) j |= 1;
      if (v < 0.f) j |= 2;
      if (v != v) j |= 4;
      if (v > FLT_MAX) j |= 8;
    }
  }
  return j;
}

// GAS/analytic_opacity.f90:3-77
void orc_analytic_opacity(int ncell, int ng, const double* wlinv, const double* temp,
                          const double* rho, int kind, double capcoef, double captpwr,
                          double caprpwr, double sigcoef, double sigtpwr, double sigrpwr,
                          double ldisp1, double ldisp2, double* gas_sig, float* gas_cap) {
  for (int i = 0; i < ncell; ++i) {
    gas_sig[i] = sigcoef * std::pow(temp[i], sigtpwr) * std::pow(rho[i], sigrpwr);
    double cc = capcoef * std::pow(temp[i], captpwr) * std::pow(rho[i], caprpwr);
    for (int ig = 1; ig <= ng; ++ig) {
      double v;
      if (kind == 1) v = cc;
      else if (kind == 2) {
        double x1 = pc_hc * wlinv[ig] / pc_kb;
        double x2 = pc_hc * wlinv[ig - 1] / pc_kb;
        v = 0.5 * cc * (x1 + x2) / sq(x1 * x2);
      } else {
        v = (ig % 2 == 1) ? cc * ldisp1 : cc * ldisp2;
      }
      gas_cap[(size_t)(ig - 1) + (size_t)ng * i] = (float)v;
    }
  }
}

// GAS/opacity_planckmean.f:17-24
void orc_opacity_planckmean(int ncell, int ng, const double* wlinv, const double* temp,
                            const float* gas_cap, double* capgrey) {
  std::vector<double> specarr(ng);
  for (int i = 0; i < ncell; ++i) {
    orc_specintv(1.0 / temp[i], wlinv, ng, ng, 1, 0, specarr.data());
    double s = 0.0;
    for (int ig = 0; ig < ng; ++ig) s = s + (double)gas_cap[(size_t)ig + (size_t)ng * i] * specarr[ig];
    capgrey[i] = s;
  }
}

// GAS/opacity_rossmean.f:17-21
void orc_opacity_rossmean(int ncell, int ng, const double* wlinv, const double* temp,
                          const double* sig, const float* gas_cap, double* capross) {
  std::vector<double> specarr(ng);
  for (int i = 0; i < ncell; ++i) {
    orc_spectintv(1.0 / temp[i], wlinv, ng, ng, 1, 0, specarr.data());
    double s = 0.0;
    for (int ig = 0; ig < ng; ++ig)
      s = s + (1.0 / (sig[i] + (double)gas_cap[(size_t)ig + (size_t)ng * i])) * specarr[ig];
    capross[i] = 1.0 / s;
  }
}

}  // extern "C"
