// oracle_transport.cpp -- the 1-D spherical hybrid IMC/DDMC particle loop of
// the reference, restated on the CPU, plus the flux and source tallies.
// TEST INFRASTRUCTURE ONLY (parity checker / timed CPU baseline).
//
// particle_advance.f90:4-327, TRANSPORT1/transport11.f90:3-515,
// TRANSPORT1/diffusion11.f90:3-633, transportmod.f:129-145,
// fluxtally.f:3-61, sourcetally.f:3-48.
//
// The DDMC per-thread group cache (groupmod.f:12-22, diffusion11.f90:95-152) is
// kept, with one deliberate difference: when the cache moves to a new cell the
// whole Planck weight array specarr(1:ng) is filled at once.  The reference
// fills it lazily under a lump mask (diffusion11.f90:274-280,564-569) and reads
// specarr(ig) of an unlumped group for doplump (:185-190) whether or not it
// was ever filled for this cell; the value used here is the one the lazy fill
// would have produced.
#include <cfloat>
#include <cstring>
#include <omp.h>
#include "oracle_internal.h"

using namespace orc;

namespace {

struct Rng {
  int mode;  // 0 mzran, 1 philox
  orc_rnd* st;
  uint64_t seed, pid;
  uint32_t k;
  double draw() {
    if (mode == 0) return mzran_real(st);
    return philox_real(seed, pid, 0u, k++);
  }
};

struct Ptcl2 {
  double dist;
  int stat;  // 0 live, 1 flux, 2 dead
  int ix, ic, ig, itype, istep, idist;
};

struct Cache {  // groupmod.f:12-22
  int ic = 0, nlump = 0;
  double capgreyinv = 0, emitlump = 0, caplump = 0, doplump = 0, speclump = 0;
  std::vector<double> specarr;
  std::vector<int> glumps;
};

struct Ctx {
  const orc_trn_in* in;
  int nx, ng;
  double X(int i) const { return in->xarr[i - 1]; }
  double VX(int i) const { return in->vxarr[i - 1]; }
  double dx(int i) const { return in->xarr[i] - in->xarr[i - 1]; }
  double dx3(int i) const { return cube(in->xarr[i]) - cube(in->xarr[i - 1]); }
  double dvdr(int i) const { return (in->vxarr[i] - in->vxarr[i - 1]) / dx(i); }
  double CAP(int ig, int ic) const { return (double)in->cap[(size_t)(ig - 1) + (size_t)ng * (ic - 1)]; }
  double SIG(int ic) const { return in->sig[ic - 1]; }
  double WL(int ig) const { return in->wl[ig - 1]; }
  double WLI(int ig) const { return in->wlinv[ig - 1]; }
  double OL(int k, int ic) const { return in->opaclump[(size_t)(k - 1) + (size_t)11 * (ic - 1)]; }
  double DIVV(int i) const { return in->divv[i - 1]; }
  double TINV(int ic) const { return in->tempinv[ic - 1]; }
  int emitgroup(double r, int ic) const {
    return orc_emitgroup(r, ic, ng, in->nep, in->nepg, in->tempinv, in->cap, in->capgrey,
                         in->emitprob, in->wlinv);
  }
};

// TRANSPORT1/transport11.f90:3-515
void transport11(const Ctx& C, orc_packet& p, Ptcl2& p2, double& vx, Rng& rng, double& eraddens,
                 double& eamp, double& jrad, double& totevelo, int& ierr) {
  const orc_trn_in* in = C.in;
  int& ix = p2.ix;
  int& ic = p2.ic;
  int& ig = p2.ig;
  double& d = p2.dist;
  double& x = p.x;
  double& mu = p.mu;
  double& e = p.e;
  double& e0 = p.e0;
  double& wl = p.wl;
  double r1, r2, db, dcol, dthm, ddop, help;
  int ixnext;
  ierr = 0;
  eraddens = 0.0;
  eamp = 0.0;
  jrad = 0.0;
  double elabfact = 1.0 - mu * vx * cinv;
  const double elabfactold = elabfact;
  const double far = 2.0 * std::fabs(std::sqrt(sq(C.X(ix + 1)) - sq(C.X(ix))));
  if (ix == 1 || mu >= -std::sqrt(1.0 - sq(C.X(ix) / x))) {
    db = std::fabs(std::sqrt(sq(C.X(ix + 1)) - (1.0 - sq(mu)) * sq(x)) - mu * x);
    ixnext = ix + 1;
  } else {
    db = std::fabs(std::sqrt(sq(C.X(ix)) - (1.0 - sq(mu)) * sq(x)) + mu * x);
    ixnext = ix - 1;
  }
  if (db != db) { ierr = 1; return; }
  if (C.SIG(ic) > 0.0) {
    r1 = rng.draw();
    dthm = -std::log(r1) / (elabfact * C.SIG(ic));
  } else {
    dthm = far;
  }
  if (C.CAP(ig, ic) <= 0.0) {
    dcol = far;
  } else {
    r1 = rng.draw();
    dcol = -std::log(r1) / (elabfact * C.CAP(ig, ic));
  }
  const double dvdr = C.dvdr(ix);
  const double vhelp = C.VX(ix) - dvdr * C.X(ix);
  double muhelp = (mu - vx * cinv) / (1.0 - mu * vx * cinv);
  if (std::fabs(vx - vhelp) / pc_c >= 0.1) {
    // Newton-Raphson Doppler distance, transport11.f90:159-199
    const double epstol = 1e-3;
    int it = 0;
    double shelp = db;
    double xhelp = std::sqrt(sq(x) + sq(shelp) + 2.0 * shelp * x * mu);
    muhelp = (mu * x + shelp) / xhelp;
    double phi = dvdr * mu * x - pc_c * (1.0 - wl * C.WLI(ig + 1)) + vhelp * muhelp + dvdr * shelp;
    double dphi = dvdr + vhelp * (1.0 - sq(muhelp)) / xhelp;
    ddop = shelp - phi / dphi;
    while ((std::fabs(ddop - shelp) > ddop * epstol) && it < 100) {
      it = it + 1;
      shelp = ddop;
      xhelp = std::sqrt(sq(x) + sq(shelp) + 2.0 * shelp * x * mu);
      muhelp = (mu * x + shelp) / xhelp;
      if (dvdr > 0.0 && ig < C.ng) {
        phi = dvdr * mu * x - pc_c * (1.0 - wl * C.WLI(ig + 1)) + vhelp * muhelp + dvdr * shelp;
      } else if (dvdr < 0.0 && ig > 1) {
        phi = dvdr * mu * x - pc_c * (1.0 - wl * C.WLI(ig)) + vhelp * muhelp + dvdr * shelp;
      } else {
        ddop = far;
        break;
      }
      dphi = dvdr + vhelp * (1.0 - sq(muhelp)) / xhelp;
      ddop = shelp - phi / dphi;
    }
    if (ddop <= 0.0 || it == 100) ddop = far;
  } else {
    if (dvdr > 0.0 && ig < C.ng) {
      ddop = 3.0 * pc_c / C.DIVV(ix) * (elabfact - wl * C.WLI(ig + 1));
    } else if (dvdr < 0.0 && ig > 1) {
      ddop = 3.0 * pc_c / C.DIVV(ix) * (elabfact - wl * C.WLI(ig));
    } else {
      ddop = far;
    }
    if (ddop < 0.0) ddop = far;
  }
  // minloc/minval over [dcol,dthm,ddop,db]; ties resolve to the first
  const double darr[4] = {dcol, dthm, ddop, db};
  int im = 0;
  for (int k = 1; k < 4; ++k)
    if (darr[k] < darr[im]) im = k;
  p2.idist = im + 1;
  d = darr[im];
  for (int k = 0; k < 4; ++k)
    if (darr[k] != darr[k]) { ierr = 3; return; }
  if (d < 0.0) { ierr = 4; return; }
  const double xold = x;
  x = std::sqrt(sq(x) + sq(d) + 2.0 * d * x * mu);
  vx = (C.VX(ix) * (C.X(ix + 1) - x) + C.VX(ix + 1) * (x - C.X(ix))) / C.dx(ix);
  if (x == 0.0) mu = 1.0;
  else mu = (xold * mu + d) / x;
  eraddens = e * sq(elabfact) * d * cinv;
  jrad = pc_c * eraddens;
  elabfact = 1.0 - mu * vx * cinv;
  if (x < C.X(1)) {
    x = C.X(1);
    vx = C.VX(1);
    ix = 1;
    ic = 1;
    r1 = rng.draw();
    mu = 1.0 - r1;
    return;
  }
  if (d == dthm || d == dcol) {
    r1 = rng.draw();
    if (d == dthm && in->thm_aniso) {
      // transport11.f90:259-281 (experimental)
      double s = std::sqrt(1.0 + 16.0 * std::pow(r1 - 0.5, 2.0));
      double mutemp = std::pow(4.0 * r1 - 2.0 + s, 1.0 / 3.0) - std::pow(s - (4.0 - 2.0 * r1), 1.0 / 3.0);
      double mh = mutemp;
      double B = 2.0 * mutemp * mh;
      double Cc = sq(mutemp) + sq(mh) - 1.0;
      double munew1 = (-B + std::sqrt(sq(B) - 4.0 * Cc)) / 2.0;
      double munew2 = (-B - std::sqrt(sq(B) - 4.0 * Cc)) / 2.0;
      bool ok1 = munew1 <= 1.0 && munew1 >= -1.0, ok2 = munew2 <= 1.0 && munew2 >= -1.0;
      if (ok1 && ok2) mu = r1 < 0.5 ? munew1 : munew2;
      else if (ok1) mu = munew1;
      else if (ok2) mu = munew2;
      else mu = 1.0 - 2.0 * r1;
    } else {
      mu = 1.0 - 2.0 * r1;
    }
    mu = (mu + vx * cinv) / (1.0 + vx * mu * cinv);
  } else if (d == db) {
    // A grazing exit through the outer edge can leave mu a rounding error
    // below 0; the reference would then index shell nx+1 (guarded here).
    bool lout = (mu >= 0.0 && ix == C.nx) || ixnext > C.nx;
    if (lout) { p2.stat = 1; return; }
  }
  if (d == dthm) {
    wl = wl * (1.0 - mu * vx * cinv) / elabfact;
    help = elabfact / (1.0 - mu * vx * cinv);
    totevelo = totevelo + e * (1.0 - help);
    e = e * help;
    e0 = e0 * help;
  } else if (d == dcol) {
    r1 = rng.draw();  // drawn and unused in the reference (transport11.f90:313)
    help = elabfact / (1.0 - mu * vx * cinv);
    totevelo = totevelo + e * (1.0 - help);
    e = e * help;
    e0 = e0 * help;
    if (C.ng != 1) {
      r1 = rng.draw();
      ig = C.emitgroup(r1, ic);
      if (((C.SIG(ic) + C.CAP(ig, ic)) * C.dx(ix) >= in->tauddmc) && !in->puretran) p2.itype = 2;
    }
    if (p2.itype == 2) {
      totevelo = totevelo + e * vx * mu * cinv;
      e = e * (1.0 - vx * mu * cinv);
      e0 = e0 * (1.0 - vx * mu * cinv);
    } else {
      r1 = rng.draw();
      wl = 1.0 / ((1.0 - r1) * C.WLI(ig) + r1 * C.WLI(ig + 1));
      wl = wl * (1.0 - vx * mu * cinv);
    }
  } else if (d == db && ixnext > ix) {
    const int l = ix + 1;
    if ((C.SIG(l) + C.CAP(ig, l)) * C.dx(ix + 1) < in->tauddmc || in->puretran) {
      x = C.X(ix + 1);
      vx = C.VX(ix + 1);
      ix = ix + 1;
      ic = ix;
    } else {
      mu = (mu - vx * cinv) / (1.0 - vx * mu * cinv);
      help = (C.CAP(ig, l) + C.SIG(l)) * C.dx(ix + 1);
      help = 4.0 / (3.0 * help + 6.0 * pc_dext);
      r1 = rng.draw();
      if (r1 < help * (1.0 + 1.5 * std::fabs(mu))) {
        p2.itype = 2;
        totevelo = totevelo + e * (1.0 - elabfact);
        e = e * elabfact;
        e0 = e0 * elabfact;
        wl = wl / elabfact;
        ix = ix + 1;
        ic = ix;
      } else {
        r1 = rng.draw();
        r2 = rng.draw();
        mu = -(r1 > r2 ? r1 : r2);
        mu = (mu + vx * cinv) / (1.0 + vx * mu * cinv);
        x = C.X(ix + 1);
        vx = C.VX(ix + 1);
      }
    }
  } else if (d == db) {
    const int l = ix - 1;
    if ((C.SIG(l) + C.CAP(ig, l)) * C.dx(ix - 1) < in->tauddmc || in->puretran) {
      x = C.X(ix);
      vx = C.VX(ix);
      ix = ix - 1;
      ic = ix;
    } else {
      mu = (mu - vx * cinv) / (1.0 - vx * mu * cinv);
      if (!in->noampfact && mu < 0.0) {
        help = 1.0 / std::fabs(mu);
        help = help < 100.0 ? help : 100.0;
        totevelo = totevelo - e * 2.0 * (0.55 * help - 1.25 * std::fabs(mu)) * vx * cinv;
        double hm2 = help - 2.0;
        eamp = e * 2.0 * 0.55 * (hm2 > 0.0 ? hm2 : 0.0) * vx * cinv;
        help = help < 2.0 ? help : 2.0;
        e0 = e0 * (1.0 + 2.0 * (0.55 * help - 1.25 * std::fabs(mu)) * vx * cinv);
        e = e * (1.0 + 2.0 * (0.55 * help - 1.25 * std::fabs(mu)) * vx * cinv);
      }
      help = (C.CAP(ig, l) + C.SIG(l)) * C.dx(ix - 1);
      help = 4.0 / (3.0 * help + 6.0 * pc_dext);
      r1 = rng.draw();
      if (r1 < help * (1.0 + 1.5 * std::fabs(mu))) {
        p2.itype = 2;
        totevelo = totevelo + e * (1.0 - elabfact);
        e = e * elabfact;
        e0 = e0 * elabfact;
        wl = wl / elabfact;
        ix = ix - 1;
        ic = ix;
      } else {
        r1 = rng.draw();
        r2 = rng.draw();
        mu = r1 > r2 ? r1 : r2;
        mu = (mu + vx * cinv) / (1.0 + vx * mu * cinv);
        x = C.X(ix);
        vx = C.VX(ix);
      }
    }
  } else if (d == ddop) {
    if (dvdr > 0.0) {
      if (ig < C.ng) {
        ig = ig + 1;
        wl = (C.WL(ig) + 1e-6 * (C.WL(ig + 1) - C.WL(ig))) * elabfactold;
      } else {
        r1 = rng.draw();
        wl = 1.0 / (r1 * C.WLI(C.ng + 1) + (1.0 - r1) * C.WLI(C.ng));
        wl = wl * elabfact;
      }
    } else if (dvdr < 0.0) {
      if (ig > 1) {
        wl = (C.WL(ig) + 1e-6 * (C.WL(ig - 1) - C.WL(ig))) * elabfactold;
        ig = ig - 1;
      } else {
        r1 = rng.draw();
        wl = 1.0 / (r1 * C.WLI(1) + (1.0 - r1) * C.WLI(2));
        wl = wl * elabfact;
      }
    }
    if (((C.SIG(ic) + C.CAP(ig, ic)) * C.dx(ix) >= in->tauddmc) && !in->puretran) {
      p2.itype = 2;
      totevelo = totevelo + e * vx * mu * cinv;
      e = e * elabfact;
      e0 = e0 * elabfact;
      wl = wl / elabfact;
    }
  } else {
    ierr = 17;
    return;
  }
}

// TRANSPORT1/diffusion11.f90:3-633 (LTE)
void diffusion11(const Ctx& C, orc_packet& p, Ptcl2& p2, double& vx, Cache& cache, Rng& rng,
                 double& eraddens, double& jrad, double& totevelo, int& ierr) {
  const orc_trn_in* in = C.in;
  const int ng = C.ng;
  int& ix = p2.ix;
  int& ic = p2.ic;
  int& ig = p2.ig;
  double& x = p.x;
  double& mu = p.mu;
  double& e = p.e;
  double& e0 = p.e0;
  double& wl = p.wl;
  double r1, r2, help, denom2, denom3;
  double emitlump, caplump, doplump;
  double opacleak[2];
  int iiig = 0, glump, l = 0;
  ierr = 0;
  eraddens = 0.0;
  jrad = 0.0;
  const double dist = C.dx(ix);
  // cache update :95-152
  if (ic != cache.ic) {
    cache.ic = ic;
    double cgi = 1.0 / in->capgrey[ic - 1];
    cache.capgreyinv = cgi > 0.0 ? cgi : 0.0;
    glump = 0;
    int gunlump = ng;
    std::fill(cache.glumps.begin(), cache.glumps.end(), 0);
    cache.speclump = C.OL(7, ic);
    if (cache.speclump == 0.0) {
      glump = 0;
    } else {
      for (int iig = 1; iig <= ng; ++iig) {
        if (C.CAP(iig, ic) * dist >= in->taulump && (C.SIG(ic) + C.CAP(iig, ic)) * dist >= in->tauddmc) {
          glump = glump + 1;
          cache.glumps[glump - 1] = iig;
        } else {
          cache.glumps[gunlump - 1] = iig;
          gunlump = gunlump - 1;
        }
      }
    }
    if (glump == ng) {
      emitlump = 1.0;
      caplump = in->capgrey[ic - 1];
      doplump = 0.0;
    } else {
      caplump = C.OL(8, ic) * cache.speclump;
      emitlump = C.OL(8, ic) * cache.capgreyinv;
      emitlump = emitlump < 1.0 ? emitlump : 1.0;
      doplump = C.OL(11, ic) * cache.speclump;
    }
    cache.nlump = glump;
    cache.emitlump = emitlump;
    cache.caplump = caplump;
    cache.doplump = doplump;
    orc_specintv(C.TINV(ic), in->wlinv, ng, ng, 1, 0, cache.specarr.data());
  }
  const double speclump = cache.speclump;
  const double capgreyinv = cache.capgreyinv;
  glump = (C.CAP(ig, ic) * dist >= in->taulump) ? cache.nlump : 0;
  if ((C.SIG(ic) + C.CAP(ig, ic)) * dist < in->tauddmc) { ierr = 100; return; }
  if (glump > 0) {
    emitlump = cache.emitlump;
    caplump = cache.caplump;
    doplump = cache.doplump;
  } else {
    emitlump = orc_specint0(C.TINV(ic), in->wlinv, ig) * capgreyinv * C.CAP(ig, ic);
    caplump = C.CAP(ig, ic);
    if (ig != ng && C.DIVV(ix) >= 0.0) {
      doplump = orc_dopspeccalc(C.TINV(ic), in->wlinv, ig) * C.DIVV(ix) /
                (cache.specarr[ig - 1] * 3.0 * pc_c);
    } else if (ig != 1 && C.DIVV(ix) < 0.0) {
      doplump = -1.0 * orc_dopspeccalc(C.TINV(ic), in->wlinv, ig - 1) * C.DIVV(ix) /
                (cache.specarr[ig - 1] * 3.0 * pc_c);
    } else {
      doplump = 0.0;
    }
  }
  if (glump > 0) {
    opacleak[0] = C.OL(1, ic);
    opacleak[1] = C.OL(2, ic);
  } else {
    if (ix != 1) l = ix - 1;
    if (ix == 1) {
      opacleak[0] = 0.0;
    } else if ((C.CAP(ig, l) + C.SIG(l)) * C.dx(ix - 1) < in->tauddmc) {
      double mfphelp = (C.CAP(ig, ic) + C.SIG(ic)) * C.dx(ix);
      double ppl = 4.0 / (3.0 * mfphelp + 6.0 * pc_dext);
      opacleak[0] = 1.5 * ppl * sq(C.X(ix)) / C.dx3(ix);
    } else {
      double mfphelp = (C.SIG(ic) + C.CAP(ig, ic)) * C.dx(ix) + (C.SIG(l) + C.CAP(ig, l)) * C.dx(ix - 1);
      opacleak[0] = 2.0 * sq(C.X(ix)) / (mfphelp * C.dx3(ix));
    }
    bool lhelp;
    if (ix == C.nx) {
      lhelp = true;
    } else {
      l = ix + 1;
      lhelp = (C.CAP(ig, l) + C.SIG(l)) * C.dx(ix + 1) < in->tauddmc;
    }
    if (lhelp) {
      double mfphelp = (C.CAP(ig, ic) + C.SIG(ic)) * C.dx(ix);
      double ppr = 4.0 / (3.0 * mfphelp + 6.0 * pc_dext);
      opacleak[1] = 1.5 * ppr * sq(C.X(ix + 1)) / C.dx3(ix);
    } else {
      double mfphelp = (C.SIG(ic) + C.CAP(ig, ic)) * C.dx(ix) + (C.SIG(l) + C.CAP(ig, l)) * C.dx(ix + 1);
      opacleak[1] = 2.0 * sq(C.X(ix + 1)) / (mfphelp * C.dx3(ix));
    }
  }
  double denom = (opacleak[0] + opacleak[1]) + (1.0 - emitlump) * caplump + doplump;
  denom = 1.0 / denom;
  r1 = rng.draw();
  const double ddmct = std::fabs(std::log(r1) * denom * cinv);
  eraddens = e * ddmct;
  jrad = pc_c * eraddens;
  r1 = rng.draw();
  const double probleak0 = opacleak[0] * denom, probleak1 = opacleak[1] * denom;
  const double pa = 0.0;
  const double pdop = doplump * denom;
  const int* glumps = cache.glumps.data();
  const double* specarr = cache.specarr.data();
  if (r1 >= pa && r1 < pa + pdop) {
    // Doppler shift :283-355
    if (glump == 0) {
      iiig = ig;
    } else {
      r1 = rng.draw();
      denom2 = 0.0;
      help = 1.0 / doplump;
      if (C.DIVV(ix) >= 0.0) {
        for (int iig = 1; iig <= glump; ++iig) {
          iiig = glumps[iig - 1];
          if (iiig == ng) continue;
          if (C.CAP(iiig + 1, ic) * dist >= in->taulump) continue;
          double resdopleak = orc_dopspeccalc(C.TINV(ic), in->wlinv, iiig) * C.DIVV(ix) / (3.0 * pc_c);
          denom2 = denom2 + resdopleak * speclump * help;
          if (denom2 > r1) break;
        }
      } else {
        for (int iig = glump; iig >= 1; --iig) {
          iiig = glumps[iig - 1];
          if (iiig == 1) continue;
          if (C.CAP(iiig - 1, ic) * dist >= in->taulump) continue;
          double resdopleak = orc_dopspeccalc(C.TINV(ic), in->wlinv, iiig - 1) * C.DIVV(ix) / (3.0 * pc_c);
          denom2 = denom2 - resdopleak * speclump * help;
          if (denom2 > r1) break;
        }
      }
    }
    if (C.DIVV(ix) >= 0.0) {
      ig = iiig + 1;
      wl = C.WL(ig);
      ig = ig < ng ? ig : ng;
    } else {
      ig = iiig - 1;
      wl = C.WL(ig + 1);
      ig = ig > 1 ? ig : 1;
    }
    if ((C.SIG(ic) + C.CAP(ig, ic)) * dist < in->tauddmc) {
      p2.itype = 1;
      r1 = rng.draw();
      mu = 1.0 - 2.0 * r1;
      r1 = rng.draw();
      x = std::pow(r1 * cube(C.X(ix + 1)) + (1.0 - r1) * cube(C.X(ix)), third_r4);
      x = x < C.X(ix + 1) ? x : C.X(ix + 1);
      x = x > C.X(ix) ? x : C.X(ix);
      vx = (C.VX(ix) * (C.X(ix + 1) - x) + C.VX(ix + 1) * (x - C.X(ix))) / C.dx(ix);
      mu = (mu + vx * cinv) / (1.0 + vx * mu * cinv);
      wl = wl * (1.0 - vx * mu * cinv);
      help = 1.0 / (1.0 - vx * mu * cinv);
      totevelo = totevelo + e * (1.0 - help);
      e = e * help;
      e0 = e0 * help;
    }
  } else if (r1 >= pa + pdop && r1 < pa + pdop + probleak0) {
    // left leakage :358-430
    p2.idist = -3;
    if (ix == 1) return;
    l = ix - 1;
    if (glump == 0) {
      iiig = ig;
    } else {
      r1 = rng.draw();
      denom2 = 0.0;
      help = 1.0 / opacleak[0];
      for (int iig = 1; iig <= glump; ++iig) {
        iiig = glumps[iig - 1];
        double specig = specarr[iiig - 1];
        double resopacleak;
        if ((C.CAP(iiig, l) + C.SIG(l)) * C.dx(ix - 1) < in->tauddmc) {
          double mfphelp = (C.CAP(iiig, ic) + C.SIG(ic)) * C.dx(ix);
          double ppl = 4.0 / (3.0 * mfphelp + 6.0 * pc_dext);
          resopacleak = 1.5 * ppl * sq(C.X(ix)) / C.dx3(ix);
        } else {
          double mfphelp = (C.SIG(ic) + C.CAP(iiig, ic)) * C.dx(ix) + (C.SIG(l) + C.CAP(iiig, l)) * C.dx(ix - 1);
          resopacleak = 2.0 * sq(C.X(ix)) / (mfphelp * C.dx3(ix));
        }
        denom2 = denom2 + specig * resopacleak * speclump * help;
        if (denom2 > r1) break;
      }
    }
    if ((C.SIG(l) + C.CAP(iiig, l)) * C.dx(ix - 1) < in->tauddmc) {
      p2.itype = 1;
      r1 = rng.draw();
      wl = 1.0 / (r1 * C.WLI(iiig + 1) + (1.0 - r1) * C.WLI(iiig));
      x = C.X(ix);
      vx = C.VX(ix);
      r1 = rng.draw();
      r2 = rng.draw();
      mu = -(r1 > r2 ? r1 : r2);
      mu = (mu + vx * cinv) / (1.0 + vx * mu * cinv);
      help = 1.0 / (1.0 - vx * mu * cinv);
      totevelo = totevelo + e * (1.0 - help);
      e = e * help;
      e0 = e0 * help;
      wl = wl * (1.0 - vx * mu * cinv);
    }
    ix = ix - 1;
    ic = ix;
    ig = iiig;
  } else if (r1 >= pa + pdop + probleak0 && r1 < pa + pdop + (probleak0 + probleak1)) {
    // right leakage :434-545
    p2.idist = -4;
    if (ix == C.nx) {
      p2.stat = 1;
      r1 = rng.draw();
      r2 = rng.draw();
      mu = r1 > r2 ? r1 : r2;
      if (glump != 0) {
        r1 = rng.draw();
        denom2 = 0.0;
        help = 1.0 / opacleak[1];
        for (int iig = 1; iig <= glump; ++iig) {
          iiig = glumps[iig - 1];
          double specig = specarr[iiig - 1];
          double mfphelp = (C.CAP(iiig, ic) + C.SIG(ic)) * C.dx(ix);
          double ppr = 4.0 / (3.0 * mfphelp + 6.0 * pc_dext);
          double resopacleak = 1.5 * ppr * sq(C.X(ix + 1)) / C.dx3(ix);
          denom2 = denom2 + specig * resopacleak * speclump * help;
          if (denom2 > r1) break;
        }
        ig = iiig;
      }
      r1 = rng.draw();
      wl = 1.0 / (r1 * C.WLI(ig + 1) + (1.0 - r1) * C.WLI(ig));
      x = C.X(C.nx + 1);
      vx = C.VX(C.nx + 1);
      mu = (mu + vx * cinv) / (1.0 + vx * mu * cinv);
      mu = mu < 1.0 ? mu : 1.0;
      help = 1.0 / (1.0 - mu * vx * cinv);
      totevelo = totevelo + e * (1.0 - help);
      wl = wl / help;
      e = e * help;
      e0 = e0 * help;
      return;
    }
    l = ix + 1;
    if (glump == 0) {
      iiig = ig;
    } else {
      r1 = rng.draw();
      denom2 = 0.0;
      help = 1.0 / opacleak[1];
      for (int iig = 1; iig <= glump; ++iig) {
        iiig = glumps[iig - 1];
        double specig = specarr[iiig - 1];
        double resopacleak;
        if ((C.CAP(iiig, l) + C.SIG(l)) * C.dx(ix + 1) < in->tauddmc) {
          double mfphelp = (C.CAP(iiig, ic) + C.SIG(ic)) * C.dx(ix);
          double ppr = 4.0 / (3.0 * mfphelp + 6.0 * pc_dext);
          resopacleak = 1.5 * ppr * sq(C.X(ix + 1)) / C.dx3(ix);
        } else {
          double mfphelp = (C.SIG(ic) + C.CAP(iiig, ic)) * C.dx(ix) + (C.SIG(l) + C.CAP(iiig, l)) * C.dx(ix + 1);
          resopacleak = 2.0 * sq(C.X(ix + 1)) / (mfphelp * C.dx3(ix));
        }
        denom2 = denom2 + specig * resopacleak * speclump * help;
        if (denom2 > r1) break;
      }
    }
    if ((C.SIG(l) + C.CAP(iiig, l)) * C.dx(ix + 1) < in->tauddmc) {
      p2.itype = 1;
      r1 = rng.draw();
      wl = 1.0 / (r1 * C.WLI(iiig + 1) + (1.0 - r1) * C.WLI(iiig));
      x = C.X(ix + 1);
      vx = C.VX(ix + 1);
      r1 = rng.draw();
      r2 = rng.draw();
      mu = r1 > r2 ? r1 : r2;
      mu = (mu + vx * cinv) / (1.0 + vx * mu * cinv);
      help = 1.0 / (1.0 - vx * mu * cinv);
      totevelo = totevelo + e * (1.0 - help);
      e = e * help;
      e0 = e0 * help;
      wl = wl * (1.0 - vx * mu * cinv);
    }
    ix = ix + 1;
    ic = ix;
    ig = iiig;
  } else {
    // effective scattering :549-620
    p2.idist = -2;
    if (glump == ng) { ierr = 102; return; }
    if (glump == 0) {
      r1 = rng.draw();
      iiig = C.emitgroup(r1, ic);
    } else {
      r1 = rng.draw();
      denom2 = 1.0 / (1.0 - emitlump);
      denom3 = 0.0;
      for (int iig = ng; iig >= glump + 1; --iig) {
        iiig = glumps[iig - 1];
        help = specarr[iiig - 1] * C.CAP(iiig, ic) * capgreyinv;
        denom3 = denom3 + help * denom2;
        if (denom3 > r1) break;
      }
    }
    ig = iiig;
    if ((C.SIG(ic) + C.CAP(ig, ic)) * dist < in->tauddmc) {
      p2.itype = 1;
      r1 = rng.draw();
      wl = 1.0 / ((1.0 - r1) * C.WLI(ig) + r1 * C.WLI(ig + 1));
      r1 = rng.draw();
      mu = 1.0 - 2.0 * r1;
      r1 = rng.draw();
      x = std::pow(r1 * cube(C.X(ix + 1)) + (1.0 - r1) * cube(C.X(ix)), third_r4);
      x = x < C.X(ix + 1) ? x : C.X(ix + 1);
      x = x > C.X(ix) ? x : C.X(ix);
      vx = (C.VX(ix) * (C.X(ix + 1) - x) + C.VX(ix + 1) * (x - C.X(ix))) / C.dx(ix);
      mu = (mu + vx * cinv) / (1.0 + vx * mu * cinv);
      help = 1.0 / (1.0 - vx * mu * cinv);
      totevelo = totevelo + e * (1.0 - help);
      e = e * help;
      e0 = e0 * help;
      wl = wl * (1.0 - vx * mu * cinv);
    }
  }
  if (x < C.X(1)) { p2.stat = 2; return; }
  totevelo = totevelo + e * (1.0 - std::exp(-C.DIVV(ix) * ddmct / 3.0));
  e = e * std::exp(-C.DIVV(ix) * ddmct / 3.0);
  e0 = e0 * std::exp(-C.DIVV(ix) * ddmct / 3.0);
}

inline uint64_t fnv_mix(uint64_t h, int32_t v) {
  uint32_t u = (uint32_t)v;
  for (int b = 0; b < 4; ++b) {
    h ^= (u >> (8 * b)) & 0xffu;
    h *= 1099511628211ull;
  }
  return h;
}

}  // namespace

extern "C" {

int orc_particle_advance(const orc_trn_in* in, orc_packet* prt, int32_t* isvacant, int64_t npart,
                         int rngmode, uint64_t seed, int nthreads, orc_rnd* rnd_states,
                         orc_trn_out* out, uint64_t* trace_hash, int32_t* trace_nstep) {
  const int nx = in->nx, ng = in->ng;
  Ctx C{in, nx, ng};
  if (nthreads < 1) nthreads = 1;
  std::memset(out->tally, 0, sizeof(double) * nx);
  std::memset(out->jrad, 0, sizeof(double) * (size_t)nx * ng);
  std::memset(out->eamp, 0, sizeof(double) * nx);
  if (in->dogrdtally && out->methodswap) std::memset(out->methodswap, 0, sizeof(int32_t) * nx);
  out->npckt = out->nflux = out->nstepimc = out->nstepddmc = out->nmethodswap = out->nstepmax = 0;
  for (int k = 0; k < 11; ++k) out->ndist[k] = 0;
  out->nposwarn = 0;
  out->ierr = 0;
  out->ierr_part = 0;

  struct Local {
    std::vector<double> tally, jrad, eamp;
    std::vector<int32_t> methodswap;
    double evelo = 0, eout = 0, sflux = 0;
    int64_t npckt = 0, nflux = 0, nimc = 0, nddmc = 0, nswap = 0, nmax = 0, ndist[11] = {0}, nwarn = 0;
    int32_t ierr = 0;
    int64_t ierr_part = 0;
  };
  std::vector<Local> loc(nthreads);

#pragma omp parallel num_threads(nthreads)
  {
    const int iomp = omp_get_thread_num();
    Local& L = loc[iomp];
    L.tally.assign(nx, 0.0);
    L.jrad.assign((size_t)nx * ng, 0.0);
    L.eamp.assign(nx, 0.0);
    L.methodswap.assign(nx, 0);
    Rng rng{rngmode, rngmode == 0 ? &rnd_states[iomp] : nullptr, seed, 0, 0};
    Cache cache;
    cache.specarr.assign(ng, 0.0);
    cache.glumps.assign(ng, 0);
#pragma omp for schedule(static, 1)
    for (int64_t ipart = 1; ipart <= npart; ++ipart) {
      if (isvacant[ipart - 1]) continue;
      orc_packet p = prt[ipart - 1];
      Ptcl2 p2{};
      rng.pid = (uint64_t)(ipart - 1);
      rng.k = 0;
      L.npckt++;
      p2.ix = orc::binsrch(p.x, in->xarr, nx + 1, false);
      p2.ic = p2.ix;
      p2.ig = orc::binsrch(p.wl, in->wl, ng + 1, false);
      if (p2.ix < 1 || p2.ig < 1) {  // NaN position or wavelength (library code 1002)
        if (in->errorfatal && L.ierr == 0) { L.ierr = 1002; L.ierr_part = ipart; }
        isvacant[ipart - 1] = 1;
        continue;
      }
      const double help = C.dx(p2.ix);
      const double tau = (C.SIG(p2.ic) + C.CAP(p2.ig, p2.ic)) * help;
      p2.itype = (in->puretran || tau < in->tauddmc) ? 1 : 2;
      double vx = (C.VX(p2.ix) * (C.X(p2.ix + 1) - p.x) + C.VX(p2.ix + 1) * (p.x - C.X(p2.ix))) /
                  (C.X(p2.ix + 1) - C.X(p2.ix));
      if (p2.itype == 1) {
        const double labfact = 1.0 - vx * p.mu / pc_c;
        p.wl = p.wl * labfact;
        p.e = p.e / labfact;
        p.e0 = p.e0 / labfact;
      }
      p2.istep = 0;
      p2.idist = 0;
      p2.stat = 0;
      uint64_t h = 1469598103934665603ull;
      while (p2.stat == 0) {
        p2.istep++;
        const int icold = p2.ic, igold = p2.ig;
        double eraddens = 0, eamp = 0, jrad = 0;
        int ierr = 0;
        if (p2.itype == 1 || in->puretran) {
          L.nimc++;
          transport11(C, p, p2, vx, rng, eraddens, eamp, jrad, L.evelo, ierr);
          if (p2.itype != 1) {
            L.nswap++;
            if (in->dogrdtally) L.methodswap[icold - 1]++;
          }
          if (!in->noampfact) L.eamp[icold - 1] += eamp;
        } else {
          L.nddmc++;
          diffusion11(C, p, p2, vx, cache, rng, eraddens, jrad, L.evelo, ierr);
          if (p2.itype == 1) {
            L.nswap++;
            if (in->dogrdtally) L.methodswap[icold - 1]++;
          }
        }
        int id = p2.idist > -3 ? p2.idist : -3;
        L.ndist[id + 3]++;
        L.tally[icold - 1] += eraddens;
        L.jrad[(size_t)(igold - 1) + (size_t)ng * (icold - 1)] += jrad;
        if (trace_hash) {
          h = fnv_mix(h, p2.idist);
          h = fnv_mix(h, p2.itype);
          h = fnv_mix(h, p2.ic);
          h = fnv_mix(h, p2.ig);
          h = fnv_mix(h, p2.stat);
        }
        if (p2.itype == 1 && p2.stat == 0) {
          if (p.x > C.X(p2.ix + 1) || p.x < C.X(p2.ix) || p.x != p.x) {
            if (ierr == 0) ierr = -99;
          }
        }
        if (ierr == -99) L.nwarn++;
        if (ierr == 0 && in->max_steps > 0 && p2.istep >= in->max_steps && p2.stat == 0)
          ierr = 1001;  // library step guard
        if (ierr > 0) {
          if (in->errorfatal && L.ierr == 0) { L.ierr = ierr; L.ierr_part = ipart; }
          p2.stat = 2;
          break;
        }
      }
      if (p2.istep > L.nmax) L.nmax = p2.istep;
      if (trace_hash) trace_hash[ipart - 1] = h;
      if (trace_nstep) trace_nstep[ipart - 1] = p2.istep;
      if (p2.stat == 2) {
        isvacant[ipart - 1] = 1;
      } else {
        L.nflux++;
        L.sflux = L.sflux - p.e;
        L.eout = L.eout + p.e;
        p.x = DBL_MAX;
        prt[ipart - 1] = p;
      }
    }
  }
  // reduction over threads in thread order
  for (int t = 0; t < nthreads; ++t) {
    const Local& L = loc[t];
    for (int i = 0; i < nx; ++i) {
      out->tally[i] += L.tally[i];
      out->eamp[i] += L.eamp[i];
      if (in->dogrdtally && out->methodswap) out->methodswap[i] += L.methodswap[i];
    }
    for (size_t k = 0; k < (size_t)nx * ng; ++k) out->jrad[k] += L.jrad[k];
    out->tot_evelo += L.evelo;
    out->tot_eout += L.eout;
    out->tot_sflux += L.sflux;
    out->npckt += L.npckt;
    out->nflux += L.nflux;
    out->nstepimc += L.nimc;
    out->nstepddmc += L.nddmc;
    out->nmethodswap += L.nswap;
    if (L.nmax > out->nstepmax) out->nstepmax = L.nmax;
    for (int k = 0; k < 11; ++k) out->ndist[k] += L.ndist[k];
    out->nposwarn += L.nwarn;
    if (L.ierr != 0 && (out->ierr == 0 || L.ierr_part < out->ierr_part)) {
      out->ierr = L.ierr;
      out->ierr_part = (int32_t)L.ierr_part;
    }
  }
  return out->ierr;
}

// fluxtally.f:30-54
void orc_fluxtally(int64_t npart, const orc_packet* prt, int32_t* isvacant, int flx_ng,
                   const double* flx_wl, double* luminos, double* lumdev, int32_t* lumnum) {
  for (int g = 0; g < flx_ng; ++g) { luminos[g] = 0.0; lumdev[g] = 0.0; lumnum[g] = 0; }
  for (int64_t ip = 0; ip < npart; ++ip) {
    if (isvacant[ip]) continue;
    const orc_packet& p = prt[ip];
    if (p.x != DBL_MAX) continue;
    int ig = orc::binsrch(p.wl, flx_wl, flx_ng + 1, false);
    if (ig < 1) continue;  // NaN wavelength (the reference indexes out of bounds)
    luminos[ig - 1] = luminos[ig - 1] + p.e;
    lumdev[ig - 1] = lumdev[ig - 1] + sq(p.e);
    lumnum[ig - 1] = lumnum[ig - 1] + 1;
    isvacant[ip] = 1;
  }
}

// sourcetally.f:24-45.  The reference checks `ic>grp_ng` where `ig>grp_ng`
// is meant (sourcetally.f:301); the intended check is made here.
int orc_sourcetally(int64_t npart, const orc_packet* prt, const int32_t* isvacant, int nx, int ng,
                    const double* xarr, const double* wl, double* src_energy, int32_t* src_number) {
  for (size_t k = 0; k < (size_t)nx * ng; ++k) { src_energy[k] = 0.0; src_number[k] = 0; }
  for (int64_t ip = 0; ip < npart; ++ip) {
    if (isvacant[ip]) continue;
    const orc_packet& p = prt[ip];
    int ig = orc::binsrch(p.wl, wl, ng + 1, false);
    int ix = orc::binsrch(p.x, xarr, nx + 1, false);
    int ic = ix;
    if (ic < 1 || ic > nx) return 1;
    if (ig < 1 || ig > ng) return 2;
    src_energy[(size_t)(ic - 1) + (size_t)nx * (ig - 1)] += p.e;
    src_number[(size_t)(ic - 1) + (size_t)nx * (ig - 1)] += 1;
  }
  return 0;
}

}  // extern "C"
