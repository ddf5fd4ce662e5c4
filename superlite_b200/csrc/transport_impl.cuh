// transport_impl.cuh -- device bodies of one IMC event (transport11) and one
// DDMC event (diffusion11) on a particle held in registers.
//
// Reference: TRANSPORT1/transport11.f90:3-515, TRANSPORT1/diffusion11.f90:3-633,
// GRID/emitgroup.f:3-54.  Arithmetic follows the Fortran expression order;
// the resolved-group scans of diffusion11 and the within-bin walk of
// emitgroup are binary searches over the per-cell running sums built by
// cell_tables_kernel (grid.cu), which hold the very partial sums the scans
// would form.
#pragma once
#include "slg_device.cuh"
#include "slg_internal.h"

namespace slg {

struct TrnArgs {
  int nx, ng, nep, nepg;
  const double *xarr, *vxarr, *divv, *wl, *wlinv, *tempinv, *sig, *capgrey, *emitprob, *opaclump;
  const float* cap;
  double tauddmc, taulump;
  int puretran, noampfact, errorfatal, thm_aniso, dogrdtally;
  long long max_steps;
  CellTables T;
  slg_packet* prt;
  int32_t* isvacant;
  long long npart;
  uint64_t seed;
  double *tally, *jrad, *eamp;
  int32_t* methodswap;
  TransportAcc* acc;
  uint64_t* trace_hash;
  int32_t* trace_nstep;
  const unsigned long long* epoch = nullptr;  // replay counter of a captured graph
  int nmodel = 1;                             // models (read by the mixed-precision kernel)
  int smem_cells = 0;                         // tally cells kept in shared memory (mixed kernel; 0: global)
  const ModelDesc* models = nullptr;
  const MixCell* mcell = nullptr;  // per-cell records (mixed-precision kernel)
  // mixed-precision kernel: per (cell, group) DDMC branch rates of an unlumped
  // group, {doplump, opacleak(1), opacleak(2), (1 - emitlump) caplump}, with
  // sentinels and neighbour flags (see mix_rate_kernel); per cell the emission
  // CDF over groups divided by capgrey, and its guide table (T.guide_m + 1
  // entries per cell)
  const float4* mrate = nullptr;
  const float* emit32 = nullptr;
  const int16_t* eguide = nullptr;
};

struct Ptcl {
  double x, mu, e, e0, wl, vx, dist;
  int ix, ig, itype, stat, idist;  // ic == ix (1-D, no void cells)
};

// The particle's model: shells nx, first cell co (0-based over every model's
// cells), first shell edge xo of xarr/vxarr.  A one-model grid is {A.nx, 0, 0}.
// ix/ic inside the event bodies stay 1-based shells of the particle's model;
// per-cell arrays are read at co + ic, edges at xo + ix.
struct MView {
  int nx, co, xo;
};

// first_gt: first position q in [0,n) with a[q] > r, else n-1 (the last
// position a linear scan visits).  a is non-decreasing, so the count of
// entries <= r is a prefix; an 8-ary search issues the 7 probes of a round
// together, which needs 4 dependent rounds of loads for n = 2000 instead of
// 11.  first_gt_range: the same when the answer is known to lie in [lo, hi].
__device__ inline int first_gt_range(const double* __restrict__ a, int lo, int hi, int n, double r) {
  while (hi - lo > 8) {
    const int step = (hi - lo) >> 3;
    double v[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) v[j] = __ldg(a + lo + (j + 1) * step);
    int c = 0;
#pragma unroll
    for (int j = 0; j < 7; ++j) c += v[j] <= r;
    const int nlo = c == 0 ? lo : lo + c * step + 1;
    const int nhi = c == 7 ? hi : lo + (c + 1) * step;
    lo = nlo;
    hi = nhi;
  }
  double v[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) v[j] = lo + j < hi ? __ldg(a + lo + j) : 0.0;
  int c = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) c += (lo + j < hi) && v[j] <= r;
  const int q = lo + c;
  return q < n ? q : n - 1;
}
__device__ inline int first_gt(const double* __restrict__ a, int n, double r) {
  return first_gt_range(a, 0, n, n, r);
}

// first_gt over running-sum table `table` (0 dop, 1 left, 2 right, 3 scat) of
// cell `cell` (0-based over all models), narrowed by the cell's guide table:
// the same answer, after one guide load and a search of about n/guide_m entries.
__device__ inline int cdf_search(const CellTables& T, int table, int cell, const double* __restrict__ a, int n,
                                 double r) {
  if (!T.guide) return first_gt(a, n, r);
  const int16_t* g = T.guide + ((size_t)cell * 4 + table) * (T.guide_m + 1);
  const int k = (int)(r * (double)T.guide_m);  // exact: guide_m is a power of two and r < 1
  return first_gt_range(a, g[k], g[k + 1], n, r);
}

// FP32 forms of first_gt_range / cdf_search (mixed-precision loop): the
// same guide narrows the search over the FP32 running sums.  Where rounding
// to FP32 moves a sum across r the answer may differ from the FP64 search by
// one position (the result stays within the guide's range).
__device__ inline int first_gt_range32(const float* __restrict__ a, int lo, int hi, int n, float r) {
  while (hi - lo > 8) {
    const int step = (hi - lo) >> 3;
    float v[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) v[j] = __ldg(a + lo + (j + 1) * step);
    int c = 0;
#pragma unroll
    for (int j = 0; j < 7; ++j) c += v[j] <= r;
    const int nlo = c == 0 ? lo : lo + c * step + 1;
    const int nhi = c == 7 ? hi : lo + (c + 1) * step;
    lo = nlo;
    hi = nhi;
  }
  float v[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) v[j] = lo + j < hi ? __ldg(a + lo + j) : 0.0f;
  int c = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) c += (lo + j < hi) && v[j] <= r;
  const int q = lo + c;
  return q < n ? q : n - 1;
}
__device__ inline int cdf_search32(const CellTables& T, int table, int cell, const float* __restrict__ a, int n,
                                   float r) {
  if (!T.guide) return first_gt_range32(a, 0, n, n, r);
  const int16_t* g = T.guide + ((size_t)cell * 4 + table) * (T.guide_m + 1);
  const int k = (int)(r * (float)T.guide_m);  // exact: guide_m is a power of two and r < 1
  return first_gt_range32(a, g[k], g[k + 1], n, r);
}

__device__ inline double CAPd(const TrnArgs& A, int ig, int ic) {
  return (double)__ldg(A.cap + (size_t)(ic - 1) * A.ng + (ig - 1));
}
__device__ inline double dxd(const TrnArgs& A, int i) { return A.xarr[i] - A.xarr[i - 1]; }
__device__ inline double dxv(const double* X, int i) { return X[i] - X[i - 1]; }

// GRID/emitgroup.f:3-54 (LTE); ic 1-based.
__device__ inline int emitgroup_dev(const TrnArgs& A, double r, int ic) {
  const double* ep = A.emitprob + (size_t)A.nep * (ic - 1);
  const double r1 = r * A.capgrey[ic - 1];
  int iep = binsrch(r1, ep, A.nep, true);
  if (iep < 0) iep = 0;
  const int ig0 = iep * A.nepg + 1;
  const int igp1 = min(ig0 + A.nepg - 1, A.ng);
  if (ig0 > igp1 - 1) return min(ig0, A.ng);
  const double* ec = A.T.emitcum + (size_t)(ic - 1) * A.ng + (ig0 - 1);
  const int n = igp1 - ig0;  // candidates ig0 .. igp1-1
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ec[mid] > r1) hi = mid;
    else lo = mid + 1;
  }
  return lo < n ? ig0 + lo : igp1;
}

// One IMC event, transport11.f90:3-515.
template <class RNG>
__device__ inline void transport11_dev(const TrnArgs& A, const MView& v, Ptcl& p, RNG& rng, double& eraddens,
                                       double& eamp, double& jrad, double& totevelo, int& ierr) {
  int& ix = p.ix;
  int& ig = p.ig;
  double& x = p.x;
  double& mu = p.mu;
  double& e = p.e;
  double& e0 = p.e0;
  double& wl = p.wl;
  double& vx = p.vx;
  const int ic = ix;
  const double* const X = A.xarr + v.xo;  // this model's shell edges
  const double* const VX = A.vxarr + v.xo;
  const int cb = v.co;                   // this model's first cell
  ierr = 0;
  eraddens = 0.0;
  eamp = 0.0;
  jrad = 0.0;
  double elabfact = 1.0 - mu * vx * cinv;
  const double elabfactold = elabfact;
  const double* sc = A.T.scal + (size_t)SCAL_N * (cb + ic - 1);
  const double far = sc[SCAL_FAR];
  const double Xa = X[ix - 1], Xb = X[ix];
  double db;
  int ixnext;
  if (ix == 1 || mu >= -sqrt(1.0 - sq(Xa / x))) {
    db = fabs(sqrt(sq(Xb) - (1.0 - sq(mu)) * sq(x)) - mu * x);
    ixnext = ix + 1;
  } else {
    db = fabs(sqrt(sq(Xa) - (1.0 - sq(mu)) * sq(x)) + mu * x);
    ixnext = ix - 1;
  }
  if (db != db) { ierr = 1; return; }
  const double sigc = A.sig[cb + ic - 1];
  double dthm, dcol, ddop, r1, r2, help;
  if (sigc > 0.0) {
    r1 = rng.draw();
    dthm = -log(r1) / (elabfact * sigc);
  } else {
    dthm = far;
  }
  const double capc = CAPd(A, ig, cb + ic);
  if (capc <= 0.0) {
    dcol = far;
  } else {
    r1 = rng.draw();
    dcol = -log(r1) / (elabfact * capc);
  }
  const double dvdr = sc[SCAL_DVDR];
  const double vhelp = VX[ix - 1] - dvdr * Xa;
  if (fabs(vx - vhelp) / pc_c >= 0.1) {
    // Newton-Raphson Doppler distance (transport11.f90:159-199)
    const double epstol = 1e-3;
    int it = 0;
    double shelp = db;
    double xhelp = sqrt(sq(x) + sq(shelp) + 2.0 * shelp * x * mu);
    double muhelp = (mu * x + shelp) / xhelp;
    double phi = dvdr * mu * x - pc_c * (1.0 - wl * A.wlinv[ig]) + vhelp * muhelp + dvdr * shelp;
    double dphi = dvdr + vhelp * (1.0 - sq(muhelp)) / xhelp;
    ddop = shelp - phi / dphi;
    while ((fabs(ddop - shelp) > ddop * epstol) && it < 100) {
      it = it + 1;
      shelp = ddop;
      xhelp = sqrt(sq(x) + sq(shelp) + 2.0 * shelp * x * mu);
      muhelp = (mu * x + shelp) / xhelp;
      if (dvdr > 0.0 && ig < A.ng) {
        phi = dvdr * mu * x - pc_c * (1.0 - wl * A.wlinv[ig]) + vhelp * muhelp + dvdr * shelp;
      } else if (dvdr < 0.0 && ig > 1) {
        phi = dvdr * mu * x - pc_c * (1.0 - wl * A.wlinv[ig - 1]) + vhelp * muhelp + dvdr * shelp;
      } else {
        ddop = far;
        break;
      }
      dphi = dvdr + vhelp * (1.0 - sq(muhelp)) / xhelp;
      ddop = shelp - phi / dphi;
    }
    if (ddop <= 0.0 || it == 100) ddop = far;
  } else {
    if (dvdr > 0.0 && ig < A.ng) {
      ddop = 3.0 * pc_c / A.divv[cb + ix - 1] * (elabfact - wl * A.wlinv[ig]);
    } else if (dvdr < 0.0 && ig > 1) {
      ddop = 3.0 * pc_c / A.divv[cb + ix - 1] * (elabfact - wl * A.wlinv[ig - 1]);
    } else {
      ddop = far;
    }
    if (ddop < 0.0) ddop = far;
  }
  // minloc over [dcol,dthm,ddop,db]; ties resolve to the first
  double d = dcol;
  int im = 1;
  if (dthm < d) { d = dthm; im = 2; }
  if (ddop < d) { d = ddop; im = 3; }
  if (db < d) { d = db; im = 4; }
  p.idist = im;
  p.dist = d;
  if (dcol != dcol || dthm != dthm || ddop != ddop) { ierr = 3; return; }
  if (d < 0.0) { ierr = 4; return; }
  const double xold = x;
  x = sqrt(sq(x) + sq(d) + 2.0 * d * x * mu);
  vx = (VX[ix - 1] * (Xb - x) + VX[ix] * (x - Xa)) / dxv(X, ix);
  if (x == 0.0) mu = 1.0;
  else mu = (xold * mu + d) / x;
  eraddens = e * sq(elabfact) * d * cinv;
  jrad = pc_c * eraddens;
  elabfact = 1.0 - mu * vx * cinv;
  if (x < X[0]) {
    x = X[0];
    vx = VX[0];
    ix = 1;
    r1 = rng.draw();
    mu = 1.0 - r1;
    return;
  }
  if (d == dthm || d == dcol) {
    r1 = rng.draw();
    if (d == dthm && A.thm_aniso) {
      // transport11.f90:259-281 (experimental)
      const double s = sqrt(1.0 + 16.0 * pow(r1 - 0.5, 2.0));
      const double mutemp = pow(4.0 * r1 - 2.0 + s, 1.0 / 3.0) - pow(s - (4.0 - 2.0 * r1), 1.0 / 3.0);
      const double mh = mutemp;
      const double B = 2.0 * mutemp * mh;
      const double Cc = sq(mutemp) + sq(mh) - 1.0;
      const double munew1 = (-B + sqrt(sq(B) - 4.0 * Cc)) / 2.0;
      const double munew2 = (-B - sqrt(sq(B) - 4.0 * Cc)) / 2.0;
      const bool ok1 = munew1 <= 1.0 && munew1 >= -1.0, ok2 = munew2 <= 1.0 && munew2 >= -1.0;
      if (ok1 && ok2) mu = r1 < 0.5 ? munew1 : munew2;
      else if (ok1) mu = munew1;
      else if (ok2) mu = munew2;
      else mu = 1.0 - 2.0 * r1;
    } else {
      mu = 1.0 - 2.0 * r1;
    }
    mu = (mu + vx * cinv) / (1.0 + vx * mu * cinv);
  } else if (d == db) {
    // transport11.f90:290-295.  A grazing exit through the outer edge can leave
    // mu a rounding error below 0; the reference would then index shell nx+1.
    if ((mu >= 0.0 && ix == v.nx) || ixnext > v.nx) { p.stat = 1; return; }
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
    if (A.ng != 1) {
      r1 = rng.draw();
      ig = emitgroup_dev(A, r1, cb + ic);
      if (((sigc + CAPd(A, ig, cb + ic)) * dxv(X, ix) >= A.tauddmc) && !A.puretran) p.itype = 2;
    }
    if (p.itype == 2) {
      totevelo = totevelo + e * vx * mu * cinv;
      e = e * (1.0 - vx * mu * cinv);
      e0 = e0 * (1.0 - vx * mu * cinv);
    } else {
      r1 = rng.draw();
      wl = 1.0 / ((1.0 - r1) * A.wlinv[ig - 1] + r1 * A.wlinv[ig]);
      wl = wl * (1.0 - vx * mu * cinv);
    }
  } else if (d == db && ixnext > ix) {
    const int l = ix + 1;
    const double capl = CAPd(A, ig, cb + l), sigl = A.sig[cb + l - 1];
    const double dxl = dxv(X, ix + 1);
    if ((sigl + capl) * dxl < A.tauddmc || A.puretran) {
      x = X[ix];
      vx = VX[ix];
      ix = ix + 1;
    } else {
      mu = (mu - vx * cinv) / (1.0 - vx * mu * cinv);
      help = (capl + sigl) * dxl;
      help = 4.0 / (3.0 * help + 6.0 * pc_dext);
      r1 = rng.draw();
      if (r1 < help * (1.0 + 1.5 * fabs(mu))) {
        p.itype = 2;
        totevelo = totevelo + e * (1.0 - elabfact);
        e = e * elabfact;
        e0 = e0 * elabfact;
        wl = wl / elabfact;
        ix = ix + 1;
      } else {
        r1 = rng.draw();
        r2 = rng.draw();
        mu = -(r1 > r2 ? r1 : r2);
        mu = (mu + vx * cinv) / (1.0 + vx * mu * cinv);
        x = X[ix];
        vx = VX[ix];
      }
    }
  } else if (d == db) {
    const int l = ix - 1;
    const double capl = CAPd(A, ig, cb + l), sigl = A.sig[cb + l - 1];
    const double dxl = dxv(X, ix - 1);
    if ((sigl + capl) * dxl < A.tauddmc || A.puretran) {
      x = X[ix - 1];
      vx = VX[ix - 1];
      ix = ix - 1;
    } else {
      mu = (mu - vx * cinv) / (1.0 - vx * mu * cinv);
      if (!A.noampfact && mu < 0.0) {
        help = 1.0 / fabs(mu);
        help = help < 100.0 ? help : 100.0;
        totevelo = totevelo - e * 2.0 * (0.55 * help - 1.25 * fabs(mu)) * vx * cinv;
        const double hm2 = help - 2.0;
        eamp = e * 2.0 * 0.55 * (hm2 > 0.0 ? hm2 : 0.0) * vx * cinv;
        help = help < 2.0 ? help : 2.0;
        e0 = e0 * (1.0 + 2.0 * (0.55 * help - 1.25 * fabs(mu)) * vx * cinv);
        e = e * (1.0 + 2.0 * (0.55 * help - 1.25 * fabs(mu)) * vx * cinv);
      }
      help = (capl + sigl) * dxl;
      help = 4.0 / (3.0 * help + 6.0 * pc_dext);
      r1 = rng.draw();
      if (r1 < help * (1.0 + 1.5 * fabs(mu))) {
        p.itype = 2;
        totevelo = totevelo + e * (1.0 - elabfact);
        e = e * elabfact;
        e0 = e0 * elabfact;
        wl = wl / elabfact;
        ix = ix - 1;
      } else {
        r1 = rng.draw();
        r2 = rng.draw();
        mu = r1 > r2 ? r1 : r2;
        mu = (mu + vx * cinv) / (1.0 + vx * mu * cinv);
        x = X[ix - 1];
        vx = VX[ix - 1];
      }
    }
  } else if (d == ddop) {
    if (dvdr > 0.0) {
      if (ig < A.ng) {
        ig = ig + 1;
        wl = (A.wl[ig - 1] + 1e-6 * (A.wl[ig] - A.wl[ig - 1])) * elabfactold;
      } else {
        r1 = rng.draw();
        wl = 1.0 / (r1 * A.wlinv[A.ng] + (1.0 - r1) * A.wlinv[A.ng - 1]);
        wl = wl * elabfact;
      }
    } else if (dvdr < 0.0) {
      if (ig > 1) {
        wl = (A.wl[ig - 1] + 1e-6 * (A.wl[ig - 2] - A.wl[ig - 1])) * elabfactold;
        ig = ig - 1;
      } else {
        r1 = rng.draw();
        wl = 1.0 / (r1 * A.wlinv[0] + (1.0 - r1) * A.wlinv[1]);
        wl = wl * elabfact;
      }
    }
    if (((sigc + CAPd(A, ig, cb + ic)) * dxv(X, ix) >= A.tauddmc) && !A.puretran) {
      p.itype = 2;
      totevelo = totevelo + e * vx * mu * cinv;
      e = e * elabfact;
      e0 = e0 * elabfact;
      wl = wl / elabfact;
    }
  } else {
    ierr = 17;
  }
}

// One DDMC event, diffusion11.f90:3-633 (LTE).
template <class RNG>
__device__ inline void diffusion11_dev(const TrnArgs& A, const MView& v, Ptcl& p, RNG& rng, double& eraddens,
                                       double& jrad, double& totevelo, int& ierr) {
  const int ng = A.ng;
  int& ix = p.ix;
  int& ig = p.ig;
  double& x = p.x;
  double& mu = p.mu;
  double& e = p.e;
  double& e0 = p.e0;
  double& wl = p.wl;
  double& vx = p.vx;
  const int ic = ix;
  const double* const X = A.xarr + v.xo;  // this model's shell edges
  const double* const VX = A.vxarr + v.xo;
  const int cb = v.co;                   // this model's first cell
  ierr = 0;
  eraddens = 0.0;
  jrad = 0.0;
  const double Xa = X[ix - 1], Xb = X[ix];
  const double dist = Xb - Xa;
  const size_t off = (size_t)(cb + ic - 1) * ng;
  const double* sc = A.T.scal + (size_t)SCAL_N * (cb + ic - 1);
  const double dx3 = sc[SCAL_DX3];
  const double capgreyinv = sc[SCAL_CAPGREYINV];
  const double sigc = A.sig[cb + ic - 1];
  const double capc = CAPd(A, ig, cb + ic);
  const double tinv = A.tempinv[cb + ic - 1];
  const double divv = A.divv[cb + ix - 1];
  const int glump = (capc * dist >= A.taulump) ? A.T.nlump[cb + ic - 1] : 0;
  if ((sigc + capc) * dist < A.tauddmc) { ierr = 100; return; }
  double emitlump, caplump, doplump, r1, r2, help;
  double o1, o2;
  if (glump > 0) {
    emitlump = sc[SCAL_EMITLUMP];
    caplump = sc[SCAL_CAPLUMP];
    doplump = sc[SCAL_DOPLUMP];
    const double* OL = A.opaclump + (size_t)11 * (cb + ic - 1);
    o1 = OL[0];
    o2 = OL[1];
  } else {
    emitlump = specint0(tinv, A.wlinv, ig) * capgreyinv * capc;
    caplump = capc;
    const double spec_ig = A.T.specarr[off + ig - 1];
    if (ig != ng && divv >= 0.0) {
      doplump = dopspeccalc(tinv, A.wlinv, ig) * divv / (spec_ig * 3.0 * pc_c);
    } else if (ig != 1 && divv < 0.0) {
      doplump = -1.0 * dopspeccalc(tinv, A.wlinv, ig - 1) * divv / (spec_ig * 3.0 * pc_c);
    } else {
      doplump = 0.0;
    }
    if (ix == 1) {
      o1 = 0.0;
    } else {
      const int l = ix - 1;
      const double capl = CAPd(A, ig, cb + l), sigl = A.sig[cb + l - 1];
      const double dxl = Xa - X[ix - 2];
      if ((capl + sigl) * dxl < A.tauddmc) {
        const double mfphelp = (capc + sigc) * dist;
        const double ppl = 4.0 / (3.0 * mfphelp + 6.0 * pc_dext);
        o1 = 1.5 * ppl * sq(Xa) / dx3;
      } else {
        const double mfphelp = (sigc + capc) * dist + (sigl + capl) * dxl;
        o1 = 2.0 * sq(Xa) / (mfphelp * dx3);
      }
    }
    bool lhelp;
    double capl = 0.0, sigl = 0.0, dxl = 0.0;
    if (ix == v.nx) {
      lhelp = true;
    } else {
      const int l = ix + 1;
      capl = CAPd(A, ig, cb + l);
      sigl = A.sig[cb + l - 1];
      dxl = X[ix + 1] - Xb;
      lhelp = (capl + sigl) * dxl < A.tauddmc;
    }
    if (lhelp) {
      const double mfphelp = (capc + sigc) * dist;
      const double ppr = 4.0 / (3.0 * mfphelp + 6.0 * pc_dext);
      o2 = 1.5 * ppr * sq(Xb) / dx3;
    } else {
      const double mfphelp = (sigc + capc) * dist + (sigl + capl) * dxl;
      o2 = 2.0 * sq(Xb) / (mfphelp * dx3);
    }
  }
  double denom = (o1 + o2) + (1.0 - emitlump) * caplump + doplump;
  denom = 1.0 / denom;
  r1 = rng.draw();
  const double ddmct = fabs(log(r1) * denom * cinv);
  eraddens = e * ddmct;
  jrad = pc_c * eraddens;
  r1 = rng.draw();
  const double pl0 = o1 * denom, pl1 = o2 * denom;
  const double pa = 0.0;
  const double pdop = doplump * denom;
  const int16_t* glumps = A.T.glumps + off;
  int iiig;
  if (r1 >= pa && r1 < pa + pdop) {
    // Doppler shift (:283-355)
    if (glump == 0) {
      iiig = ig;
    } else {
      r1 = rng.draw();
      const int q = cdf_search(A.T, 0, cb + ic - 1, A.T.cdf_dop + off, glump, r1);
      iiig = divv >= 0.0 ? glumps[q] : glumps[glump - 1 - q];
    }
    if (divv >= 0.0) {
      ig = iiig + 1;
      wl = A.wl[ig - 1];
      ig = ig < ng ? ig : ng;
    } else {
      ig = iiig - 1;
      wl = A.wl[ig];
      ig = ig > 1 ? ig : 1;
    }
    if ((sigc + CAPd(A, ig, cb + ic)) * dist < A.tauddmc) {
      p.itype = 1;
      r1 = rng.draw();
      mu = 1.0 - 2.0 * r1;
      r1 = rng.draw();
      x = pow(r1 * cube(Xb) + (1.0 - r1) * cube(Xa), third_r4);
      x = x < Xb ? x : Xb;
      x = x > Xa ? x : Xa;
      vx = (VX[ix - 1] * (Xb - x) + VX[ix] * (x - Xa)) / dist;
      mu = (mu + vx * cinv) / (1.0 + vx * mu * cinv);
      wl = wl * (1.0 - vx * mu * cinv);
      help = 1.0 / (1.0 - vx * mu * cinv);
      totevelo = totevelo + e * (1.0 - help);
      e = e * help;
      e0 = e0 * help;
    }
  } else if (r1 >= pa + pdop && r1 < pa + pdop + (pl0 + pl1)) {
    // leakage to a neighbour: left (:358-430) or right (:434-545).  Both
    // directions run one code path (same draws, same arithmetic as each
    // branch of the reference) so lanes of a warp leaking either way stay
    // together.
    const bool right = r1 >= pa + pdop + pl0;
    p.idist = right ? -4 : -3;
    if (!right && ix == 1) return;
    if (right && ix == v.nx) {
      // escape through the outer edge (:438-478)
      p.stat = 1;
      r1 = rng.draw();
      r2 = rng.draw();
      mu = r1 > r2 ? r1 : r2;
      if (glump != 0) {
        r1 = rng.draw();
        ig = glumps[cdf_search(A.T, 2, cb + ic - 1, A.T.cdf_right + off, glump, r1)];
      }
      r1 = rng.draw();
      wl = 1.0 / (r1 * A.wlinv[ig] + (1.0 - r1) * A.wlinv[ig - 1]);
      x = X[v.nx];
      vx = VX[v.nx];
      mu = (mu + vx * cinv) / (1.0 + vx * mu * cinv);
      mu = mu < 1.0 ? mu : 1.0;
      help = 1.0 / (1.0 - mu * vx * cinv);
      totevelo = totevelo + e * (1.0 - help);
      wl = wl / help;
      e = e * help;
      e0 = e0 * help;
      return;
    }
    const int l = right ? ix + 1 : ix - 1;
    if (glump == 0) {
      iiig = ig;
    } else {
      r1 = rng.draw();
      iiig = glumps[cdf_search(A.T, right ? 2 : 1, cb + ic - 1, (right ? A.T.cdf_right : A.T.cdf_left) + off, glump, r1)];
    }
    const double dxl = right ? X[ix + 1] - Xb : Xa - X[ix - 2];
    if ((A.sig[cb + l - 1] + CAPd(A, iiig, cb + l)) * dxl < A.tauddmc) {
      p.itype = 1;
      r1 = rng.draw();
      wl = 1.0 / (r1 * A.wlinv[iiig] + (1.0 - r1) * A.wlinv[iiig - 1]);
      x = right ? Xb : Xa;
      vx = VX[right ? ix : ix - 1];
      r1 = rng.draw();
      r2 = rng.draw();
      const double m = r1 > r2 ? r1 : r2;
      mu = right ? m : -m;
      mu = (mu + vx * cinv) / (1.0 + vx * mu * cinv);
      help = 1.0 / (1.0 - vx * mu * cinv);
      totevelo = totevelo + e * (1.0 - help);
      e = e * help;
      e0 = e0 * help;
      wl = wl * (1.0 - vx * mu * cinv);
    }
    ix = l;
    ig = iiig;
  } else {
    // effective scattering (:549-620)
    p.idist = -2;
    if (glump == ng) { ierr = 102; return; }
    if (glump == 0) {
      r1 = rng.draw();
      iiig = emitgroup_dev(A, r1, cb + ic);
    } else {
      r1 = rng.draw();
      const int q = cdf_search(A.T, 3, cb + ic - 1, A.T.cdf_scat + off, ng - glump, r1);
      iiig = glumps[ng - 1 - q];
    }
    ig = iiig;
    if ((sigc + CAPd(A, ig, cb + ic)) * dist < A.tauddmc) {
      p.itype = 1;
      r1 = rng.draw();
      wl = 1.0 / ((1.0 - r1) * A.wlinv[ig - 1] + r1 * A.wlinv[ig]);
      r1 = rng.draw();
      mu = 1.0 - 2.0 * r1;
      r1 = rng.draw();
      x = pow(r1 * cube(Xb) + (1.0 - r1) * cube(Xa), third_r4);
      x = x < Xb ? x : Xb;
      x = x > Xa ? x : Xa;
      vx = (VX[ix - 1] * (Xb - x) + VX[ix] * (x - Xa)) / dist;
      mu = (mu + vx * cinv) / (1.0 + vx * mu * cinv);
      help = 1.0 / (1.0 - vx * mu * cinv);
      totevelo = totevelo + e * (1.0 - help);
      e = e * help;
      e0 = e0 * help;
      wl = wl * (1.0 - vx * mu * cinv);
    }
  }
  if (x < X[0]) { p.stat = 2; return; }
  const double dv = A.divv[cb + ix - 1];
  totevelo = totevelo + e * (1.0 - exp(-dv * ddmct / 3.0));
  e = e * exp(-dv * ddmct / 3.0);
  e0 = e0 * exp(-dv * ddmct / 3.0);
}

}  // namespace slg
