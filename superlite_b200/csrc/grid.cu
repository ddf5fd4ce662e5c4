// grid.cu -- DDMC leakage opacities, emission probabilities and the per-cell
// tables of the transport kernels, for sm_100a.
//
// Reference: GRID/leakage_opacity11.f90:3-174, GRID/emission_probability.f90:3-67,
// GRID/emitgroup.f:3-54, TRANSPORT1/diffusion11.f90:95-152 (per-thread group
// cache) and the resolved-group sampling loops of diffusion11.f90:283-584.
//
// The reference rebuilds a per-thread cache (lump list, Planck weights) every
// time a DDMC particle enters a new cell and then scans up to ng groups per
// event to sample a resolved group.  Here every cell's cache and every scan's
// running partial sums are built once per call (build_cell_tables), in the
// reference's accumulation order, so a particle's linear scan "first position
// whose running sum exceeds r" becomes a binary search over the same
// sequence of partial sums (all terms are >= 0, so the sums are monotone).
#include <cuda_runtime.h>
#include <cfloat>
#include "slg_device.cuh"
#include "slg_internal.h"

namespace slg {
namespace {

constexpr int GB = 256;  // block size of the per-cell kernels

__device__ inline double block_sum(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int w = GB / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + w];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

// CT: opacity type, float (grd_cap) or double (the FP64 opacity of the
// differentiable path).
template <class CT>
struct LeakArgsT {
  int nx, ng;
  const double *xarr, *vol, *divv, *tempinv, *sig, *wlinv;
  const CT *cap, *capemit;
  double tauddmc, taulump;
  double* opaclump;
  const int4* cellmap;  // {shell, model shells, model first cell, model} per cell; null: one model
};
using LeakArgs = LeakArgsT<float>;

// Arguments seen from cell c (0-based over all models): per-cell arrays start
// at the cell's model, nx is the model's, *i the 1-based shell in the model.
template <class CT>
__device__ inline LeakArgsT<CT> leak_view(LeakArgsT<CT> A, int c, int* i) {
  *i = c + 1;
  if (A.cellmap) {
    const int4 m = A.cellmap[c];
    const int co = m.z;
    *i = m.x;
    A.nx = m.y;
    A.xarr += co + m.w;
    A.vol += co; A.divv += co; A.tempinv += co; A.sig += co;
    A.cap += (size_t)co * A.ng;
    if (A.capemit) A.capemit += (size_t)co * A.ng;
    A.opaclump += (size_t)11 * co;
  }
  return A;
}

// leakage_opacity11.f90:30-171, one block per cell.  Sums are fixed-shape
// tree reductions (the reference sums sequentially).
template <class CT>
__global__ void __launch_bounds__(GB) leakage_kernel(const LeakArgsT<CT> A0) {
  __shared__ double sh[GB];
  __shared__ double shv[GB];
  __shared__ int shi[GB];
  int i0;
  const LeakArgsT<CT> A = leak_view(A0, blockIdx.x, &i0);
  const int i = i0;  // 1-based cell
  const int l = i, ng = A.ng;
  const double* X = A.xarr - 1;  // 1-based view
  auto dx = [&](int k) { return A.xarr[k] - A.xarr[k - 1]; };
  const CT* capl = A.cap + (size_t)(l - 1) * ng;
  const double sigl = A.sig[l - 1];
  const double dist = dx(i);
  const double tinv = A.tempinv[l - 1];
  const double hct = hck * tinv;
  const double divv = A.divv[l - 1];
  const int icnb1 = max(i - 1, 1), icnb2 = min(i + 1, A.nx);
  auto lumpable = [&](int ig) {
    const double c = (double)capl[ig - 1];
    return c * dist >= A.taulump && (sigl + c) * dist >= A.tauddmc;
  };
  // speclump
  double s = 0.0;
  for (int ig = threadIdx.x + 1; ig <= ng; ig += GB)
    if (lumpable(ig)) s = s + specintv_elem(hct, A.wlinv, ig - 1);
  double speclump = block_sum(s, sh);
  speclump = speclump > 0.0 ? 1.0 / speclump : 0.0;
  // caplump, capemitlump, igemitmax (first strict maximum over loop 1 then loop 2)
  double cl = 0.0, cel = 0.0, bestv = 0.0;
  int besto = 0x7fffffff;
  for (int ig = threadIdx.x + 1; ig <= ng; ig += GB) {
    if (!lumpable(ig)) continue;
    const double sv = specintv_elem(hct, A.wlinv, ig - 1);
    const double h1 = sv * (double)capl[ig - 1];
    cl = cl + h1;
    if (h1 > bestv || (h1 == bestv && h1 > 0.0 && ig < besto)) { bestv = h1; besto = ig; }
    const double h2 = A.capemit ? sv * (double)A.capemit[(size_t)(l - 1) * ng + ig - 1] : 0.0;
    cel = cel + h2;
    if (h2 > bestv) { bestv = h2; besto = ng + ig; }
  }
  const double caplump = block_sum(cl, sh);
  const double capemitlump = block_sum(cel, sh);
  shv[threadIdx.x] = bestv;
  shi[threadIdx.x] = besto;
  __syncthreads();
  for (int w = GB / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      const double v2 = shv[threadIdx.x + w];
      const int o2 = shi[threadIdx.x + w];
      if (v2 > shv[threadIdx.x] || (v2 == shv[threadIdx.x] && o2 < shi[threadIdx.x])) {
        shv[threadIdx.x] = v2;
        shi[threadIdx.x] = o2;
      }
    }
    __syncthreads();
  }
  int igemitmax = 0;
  if (shv[0] > 0.0) igemitmax = shi[0] > ng ? shi[0] - ng : shi[0];
  __syncthreads();
  // doplump
  double dl = 0.0;
  if (divv >= 0.0) {
    for (int ig = threadIdx.x + 1; ig <= ng - 1; ig += GB) {
      if ((double)capl[ig - 1] * dist < A.taulump) continue;
      if ((double)capl[ig] * dist >= A.taulump) continue;
      if ((sigl + (double)capl[ig - 1]) * dist < A.tauddmc) continue;
      dl = dl + dopspeccalc(tinv, A.wlinv, ig) * divv / (3.0 * pc_c);
    }
  } else {
    for (int ig = threadIdx.x + 2; ig <= ng; ig += GB) {
      if ((double)capl[ig - 1] * dist < A.taulump) continue;
      if ((double)capl[ig - 2] * dist >= A.taulump) continue;
      if ((sigl + (double)capl[ig - 1]) * dist < A.tauddmc) continue;
      dl = dl - dopspeccalc(tinv, A.wlinv, ig - 1) * divv / (3.0 * pc_c);
    }
  }
  const double doplump = block_sum(dl, sh);
  // leakage opacities
  const double vterm = 3.0 * A.vol[l - 1] / pc_pi4;
  double o1 = 0.0, o2 = 0.0;
  for (int ig = threadIdx.x + 1; ig <= ng; ig += GB) {
    if (!lumpable(ig)) continue;
    const double specval = specintv_elem(hct, A.wlinv, ig - 1);
    const double cap_l = (double)capl[ig - 1];
    bool lhelp;
    if (i == 1) lhelp = true;
    else lhelp = ((double)A.cap[(size_t)(icnb1 - 1) * ng + ig - 1] + A.sig[icnb1 - 1]) * dx(i - 1) < A.tauddmc;
    if (lhelp) {
      const double help = (cap_l + sigl) * dx(i);
      const double ppl = 4.0 / (3.0 * help + 6.0 * pc_dext);
      o1 = o1 + (specval * speclump) * 1.5 * ppl * sq(X[i]) / vterm;
    } else {
      const double help = (sigl + cap_l) * dx(i) +
                          (A.sig[icnb1 - 1] + (double)A.cap[(size_t)(icnb1 - 1) * ng + ig - 1]) * dx(i - 1);
      o1 = o1 + (specval * speclump) * 2.0 * sq(X[i]) / (help * 3.0 * A.vol[l - 1] / pc_pi4);
    }
    if (i == A.nx) lhelp = true;
    else lhelp = ((double)A.cap[(size_t)(icnb2 - 1) * ng + ig - 1] + A.sig[icnb2 - 1]) * dx(i + 1) < A.tauddmc;
    if (lhelp) {
      const double help = (cap_l + sigl) * dx(i);
      const double ppr = 4.0 / (3.0 * help + 6.0 * pc_dext);
      o2 = o2 + (specval * speclump) * 1.5 * ppr * sq(X[i + 1]) / vterm;
    } else {
      const double help = (sigl + cap_l) * dx(i) +
                          (A.sig[icnb2 - 1] + (double)A.cap[(size_t)(icnb2 - 1) * ng + ig - 1]) * dx(i + 1);
      o2 = o2 + (specval * speclump) * 2.0 * sq(X[i + 1]) / (help * 3.0 * A.vol[l - 1] / pc_pi4);
    }
  }
  const double ol1 = block_sum(o1, sh);
  const double ol2 = block_sum(o2, sh);
  if (threadIdx.x == 0) {
    double* ol = A.opaclump + (size_t)11 * (l - 1);
    ol[0] = ol1;
    ol[1] = ol2;
    ol[2] = 0.0; ol[3] = 0.0; ol[4] = 0.0; ol[5] = 0.0;
    ol[6] = speclump;
    ol[7] = caplump;
    ol[8] = capemitlump;
    ol[9] = (double)igemitmax;
    ol[10] = doplump;
  }
}

// emission_probability.f90:40-63: bin sums are sequential within a bin (one
// thread per bin) and the running sum over bins is sequential (thread 0), as in
// the reference.
__global__ void __launch_bounds__(GB) emitprob_kernel(int ng, int nep, int nepg, const double* __restrict__ tempinv,
                                                      const float* __restrict__ cap,
                                                      const double* __restrict__ capgrey,
                                                      const double* __restrict__ wlinv,
                                                      double* __restrict__ emitprob) {
  extern __shared__ double binsum[];
  const int l = blockIdx.x;
  double* ep = emitprob + (size_t)nep * l;
  if (ng == 1) {
    if (threadIdx.x == 0) ep[0] = capgrey[l];
    return;
  }
  const double hct = hck * tempinv[l];
  const float* capl = cap + (size_t)l * ng;
  for (int iep = threadIdx.x + 1; iep <= nep - 1; iep += blockDim.x) {
    const int ig = (iep - 1) * nepg + 1;
    const int top = min(iep * nepg, ng);
    double s = 0.0;
    for (int g = ig; g <= top; ++g) s = s + specintv_elem(hct, wlinv, g - 1) * (double)capl[g - 1];
    binsum[iep - 1] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double help = 0.0;
    for (int iep = 1; iep <= nep - 1; ++iep) {
      help = help + binsum[iep - 1];
      ep[iep - 1] = help;
    }
    ep[nep - 1] = capgrey[l];
  }
}

// d/dT of specintv_elem and dopspeccalc (groupmod.f:123-143, :189-198) at
// temperature T: x = hc/(lambda k T) scales as 1/T; zero where x is clamped.
__device__ inline double dspec_dT(double hct, double T, const double* __restrict__ wlinv, int g0) {
  const double x1 = hct * wlinv[g0], x2 = hct * wlinv[g0 + 1];
  const double xm = 0.5 * (x2 + x1), ax = fabs(x2 - x1);
  double dfp = 0.0;
  if (xm < 300.0) {
    const double ex = exp(xm), d = ex - 1.0;
    dfp = 3.0 * sq(xm) / d - cube(xm) * ex / sq(d);
  }
  return -(ftpi4 * ax * (fplanck(xm) + xm * dfp)) / T;
}
__device__ inline double ddop_dT(double tinv, const double* __restrict__ wlinv, int ig) {
  const double x = hck * tinv * wlinv[ig];
  if (x >= 300.0) return 0.0;
  const double ex = exp(x);
  return -dopspeccalc(tinv, wlinv, ig) * tinv * (4.0 - x * ex / (ex - 1.0));
}

__global__ void __launch_bounds__(GB, 4) leakage_bwd_kernel(const LeakArgsT<double> A0, const double* __restrict__ gol,
                                                         double* __restrict__ gcap, double* __restrict__ gsig,
                                                         double* __restrict__ gT) {
  __shared__ double sh[GB];
  const int c = blockIdx.x;  // cell over all models, 0-based
  int i0;
  const LeakArgsT<double> A = leak_view(A0, c, &i0);
  const int i = i0, ng = A.ng;
  const double* X = A.xarr - 1;
  auto dx = [&](int k) { return A.xarr[k] - A.xarr[k - 1]; };
  const double* capl = A.cap + (size_t)(i - 1) * ng;
  const double sigl = A.sig[i - 1];
  const double dist = dx(i);
  const double tinv = A.tempinv[i - 1], T = 1.0 / tinv;
  const double hct = hck * tinv;
  const double divv = A.divv[i - 1];
  const double* ol = A.opaclump + (size_t)11 * (i - 1);
  const double* u = gol + (size_t)11 * c;
  const double speclump = ol[6], ol1 = ol[0], ol2 = ol[1];
  const double u1 = u[0], u2 = u[1], u7 = u[6], u8 = u[7], u11 = u[10];
  const double vterm = 3.0 * A.vol[i - 1] / pc_pi4;
  double gs = 0.0, gt = 0.0, gsl = 0.0, gsr = 0.0;  // gsl, gsr: the neighbours' sigma, reduced once per block
  for (int ig = threadIdx.x + 1; ig <= ng; ig += GB) {
    const double cg = capl[ig - 1];
    if (!(cg * dist >= A.taulump && (sigl + cg) * dist >= A.tauddmc)) continue;
    const double sv = specintv_elem(hct, A.wlinv, ig - 1);
    // left leakage term a and d a / d(opacity sum) of this cell (da) and the left one (dal)
    double a, da, dal = 0.0;
    const bool lint = i != 1 && (A.cap[(size_t)(i - 2) * ng + ig - 1] + A.sig[i - 2]) * dx(i - 1) >= A.tauddmc;
    if (!lint) {
      const double q = 3.0 * ((cg + sigl) * dist) + 6.0 * pc_dext;
      a = 1.5 * (4.0 / q) * sq(X[i]) / vterm;
      da = -a * 3.0 / q * dist;
    } else {
      const double help = (sigl + cg) * dist + (A.sig[i - 2] + A.cap[(size_t)(i - 2) * ng + ig - 1]) * dx(i - 1);
      a = 2.0 * sq(X[i]) / (help * vterm);
      da = -a / help * dist;
      dal = -a / help * dx(i - 1);
    }
    double b, db, dbr = 0.0;
    const bool rint = i != A.nx && (A.cap[(size_t)i * ng + ig - 1] + A.sig[i]) * dx(i + 1) >= A.tauddmc;
    if (!rint) {
      const double q = 3.0 * ((cg + sigl) * dist) + 6.0 * pc_dext;
      b = 1.5 * (4.0 / q) * sq(X[i + 1]) / vterm;
      db = -b * 3.0 / q * dist;
    } else {
      const double help = (sigl + cg) * dist + (A.sig[i] + A.cap[(size_t)i * ng + ig - 1]) * dx(i + 1);
      b = 2.0 * sq(X[i + 1]) / (help * vterm);
      db = -b / help * dist;
      dbr = -b / help * dx(i + 1);
    }
    // ol1 = sum w_g a_g with w_g = sv_g speclump and speclump = 1/sum sv: d ol1/d sv_g = speclump (a_g - ol1)
    const double ua = u1 * sv * speclump, ub = u2 * sv * speclump;
    const double us = u1 * speclump * (a - ol1) + u2 * speclump * (b - ol2) - u7 * speclump * speclump + u8 * cg;
    gt += us * dspec_dT(hct, T, A.wlinv, ig - 1);
    atomicAdd(&gcap[(size_t)c * ng + ig - 1], u8 * sv + ua * da + ub * db);
    gs += ua * da + ub * db;
    if (lint) {
      atomicAdd(&gcap[(size_t)(c - 1) * ng + ig - 1], ua * dal);
      gsl += ua * dal;
    }
    if (rint) {
      atomicAdd(&gcap[(size_t)(c + 1) * ng + ig - 1], ub * dbr);
      gsr += ub * dbr;
    }
  }
  if (u11 != 0.0) {
    if (divv >= 0.0) {
      for (int ig = threadIdx.x + 1; ig <= ng - 1; ig += GB) {
        if (capl[ig - 1] * dist < A.taulump || capl[ig] * dist >= A.taulump) continue;
        if ((sigl + capl[ig - 1]) * dist < A.tauddmc) continue;
        gt += u11 * ddop_dT(tinv, A.wlinv, ig) * divv / (3.0 * pc_c);
      }
    } else {
      for (int ig = threadIdx.x + 2; ig <= ng; ig += GB) {
        if (capl[ig - 1] * dist < A.taulump || capl[ig - 2] * dist >= A.taulump) continue;
        if ((sigl + capl[ig - 1]) * dist < A.tauddmc) continue;
        gt -= u11 * ddop_dT(tinv, A.wlinv, ig - 1) * divv / (3.0 * pc_c);
      }
    }
  }
  gs = block_sum(gs, sh);
  gt = block_sum(gt, sh);
  gsl = block_sum(gsl, sh);
  gsr = block_sum(gsr, sh);
  if (threadIdx.x == 0) {
    atomicAdd(&gsig[c], gs);
    gT[c] += gt;
    if (gsl != 0.0) atomicAdd(&gsig[c - 1], gsl);
    if (gsr != 0.0) atomicAdd(&gsig[c + 1], gsr);
  }
}

struct TabArgs {
  int nx, ng, nep, nepg;
  const double *xarr, *vxarr, *divv, *wlinv, *tempinv, *sig, *capgrey, *opaclump, *emitprob;
  const float* cap;
  double tauddmc, taulump;
  CellTables T;
  const int4* cellmap = nullptr;  // as LeakArgs::cellmap
};

// Arguments seen from cell c (see leak_view); *ic is the 1-based shell.
__device__ inline TabArgs tab_view(TabArgs A, int c, int* ic) {
  *ic = c + 1;
  if (A.cellmap) {
    const int4 m = A.cellmap[c];
    const int co = m.z;
    const size_t cg = (size_t)co * A.ng;
    *ic = m.x;
    A.nx = m.y;
    A.xarr += co + m.w; A.vxarr += co + m.w;
    A.divv += co; A.tempinv += co; A.sig += co; A.capgrey += co;
    A.opaclump += (size_t)11 * co;
    A.emitprob += (size_t)A.nep * co;
    A.cap += cg;
    A.T.specarr += cg; A.T.glumps += cg; A.T.cdf_dop += cg; A.T.cdf_left += cg; A.T.cdf_right += cg;
    A.T.cdf_scat += cg; A.T.emitcum += cg;
    if (A.T.guide) A.T.guide += (size_t)co * 4 * (A.T.guide_m + 1);
    A.T.nlump += co;
    A.T.scal += (size_t)SCAL_N * co;
  }
  return A;
}

// Per-cell transport tables (see CellTables).  Phase A computes every term in
// parallel; phase B forms the running sums sequentially, one thread per table,
// in the order of the reference's loops.
__global__ void __launch_bounds__(GB) cell_tables_kernel(const TabArgs A0) {
  __shared__ int warp_l[GB / 32], warp_u[GB / 32];
  __shared__ int base_l, base_u;
  int ic0;
  const TabArgs A = tab_view(A0, blockIdx.x, &ic0);
  const int ic = ic0, ix = ic;
  const int ng = A.ng;
  const size_t off = (size_t)(ic - 1) * ng;
  const float* capc = A.cap + off;
  const double dist = A.xarr[ix] - A.xarr[ix - 1];
  const double sigc = A.sig[ic - 1];
  const double tinv = A.tempinv[ic - 1];
  const double hct = hck * tinv;
  const double* OL = A.opaclump + (size_t)11 * (ic - 1);
  const double speclump = OL[6];
  double* specarr = A.T.specarr + off;
  int16_t* glumps = A.T.glumps + off;
  // specarr and the lump ordering (diffusion11.f90:103-124)
  if (threadIdx.x == 0) { base_l = 0; base_u = 0; }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int c0 = 0; c0 < ng; c0 += GB) {
    const int ig = c0 + threadIdx.x + 1;
    bool lump = false;
    if (ig <= ng) {
      specarr[ig - 1] = specintv_elem(hct, A.wlinv, ig - 1);
      const double c = (double)capc[ig - 1];
      lump = speclump != 0.0 && c * dist >= A.taulump && (sigc + c) * dist >= A.tauddmc;
    }
    const unsigned bl = __ballot_sync(0xffffffffu, ig <= ng && lump);
    const unsigned bu = __ballot_sync(0xffffffffu, ig <= ng && !lump);
    if (lane == 0) { warp_l[wid] = __popc(bl); warp_u[wid] = __popc(bu); }
    __syncthreads();
    int pl = base_l, pu = base_u;
    for (int w = 0; w < wid; ++w) { pl += warp_l[w]; pu += warp_u[w]; }
    const unsigned below = (1u << lane) - 1u;
    pl += __popc(bl & below);
    pu += __popc(bu & below);
    if (ig <= ng) {
      if (lump) glumps[pl] = (int16_t)ig;              // glumps(pl+1)
      else if (speclump != 0.0) glumps[ng - 1 - pu] = (int16_t)ig;  // glumps(ng-pu)
      else glumps[ig - 1] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 0; w < GB / 32; ++w) { base_l += warp_l[w]; base_u += warp_u[w]; }
    }
    __syncthreads();
  }
  const int nlump = base_l;
  // scalars (diffusion11.f90:98-150)
  const double cgi0 = 1.0 / A.capgrey[ic - 1];
  const double capgreyinv = cgi0 > 0.0 ? cgi0 : 0.0;
  double emitlump, caplump, doplump;
  if (nlump == ng) {
    emitlump = 1.0;
    caplump = A.capgrey[ic - 1];
    doplump = 0.0;
  } else {
    caplump = OL[7] * speclump;
    emitlump = OL[7] * capgreyinv;
    emitlump = emitlump < 1.0 ? emitlump : 1.0;
    doplump = OL[10] * speclump;
  }
  const double X0 = A.xarr[ix - 1], X1 = A.xarr[ix];
  const double dx3 = cube(X1) - cube(X0);
  if (threadIdx.x == 0) {
    A.T.nlump[ic - 1] = nlump;
    double* sc = A.T.scal + (size_t)SCAL_N * (ic - 1);
    sc[SCAL_EMITLUMP] = emitlump;
    sc[SCAL_CAPLUMP] = caplump;
    sc[SCAL_DOPLUMP] = doplump;
    sc[SCAL_CAPGREYINV] = capgreyinv;
    sc[SCAL_SPECLUMP] = speclump;
    sc[SCAL_FAR] = 2.0 * fabs(sqrt(sq(X1) - sq(X0)));
    sc[SCAL_DX3] = dx3;
    sc[SCAL_DVDR] = (A.vxarr[ix] - A.vxarr[ix - 1]) / dist;
  }
  __syncthreads();  // glumps and specarr visible to the block
  const double divv = A.divv[ix - 1];
  double* cdop = A.T.cdf_dop + off;
  double* cleft = A.T.cdf_left + off;
  double* cright = A.T.cdf_right + off;
  double* cscat = A.T.cdf_scat + off;
  double* ecum = A.T.emitcum + off;
  // ---- phase A: terms
  if (nlump > 0) {
    const double hdop = 1.0 / doplump;
    const double hl = 1.0 / OL[0], hr = 1.0 / OL[1];
    const double denom2 = 1.0 / (1.0 - emitlump);
    for (int q = threadIdx.x + 1; q <= ng; q += GB) {
      // Doppler (diffusion11.f90:290-314): position q in loop order
      if (q <= nlump) {
        double t = 0.0;
        if (divv >= 0.0) {
          const int iiig = glumps[q - 1];
          if (!(iiig == ng) && !((double)capc[iiig] * dist >= A.taulump)) {
            const double res = dopspeccalc(tinv, A.wlinv, iiig) * divv / (3.0 * pc_c);
            t = res * speclump * hdop;
          }
        } else {
          const int iig = nlump + 1 - q;
          const int iiig = glumps[iig - 1];
          if (!(iiig == 1) && !((double)capc[iiig - 2] * dist >= A.taulump)) {
            const double res = dopspeccalc(tinv, A.wlinv, iiig - 1) * divv / (3.0 * pc_c);
            t = -(res * speclump * hdop);
          }
        }
        cdop[q - 1] = t;
        // left leak (:378-397)
        const int iiig = glumps[q - 1];
        const double specig = specarr[iiig - 1];
        const double capi = (double)capc[iiig - 1];
        if (ix > 1) {
          const int l = ix - 1;
          const double capl = (double)A.cap[(size_t)(l - 1) * ng + iiig - 1];
          const double dxl = A.xarr[ix - 1] - A.xarr[ix - 2];
          double res;
          if ((capl + A.sig[l - 1]) * dxl < A.tauddmc) {
            const double mfphelp = (capi + sigc) * dist;
            const double ppl = 4.0 / (3.0 * mfphelp + 6.0 * pc_dext);
            res = 1.5 * ppl * sq(X0) / dx3;
          } else {
            const double mfphelp = (sigc + capi) * dist + (A.sig[l - 1] + capl) * dxl;
            res = 2.0 * sq(X0) / (mfphelp * dx3);
          }
          cleft[q - 1] = specig * res * speclump * hl;
        }
        // right leak: boundary (:450-460) or interior (:492-511)
        double res;
        if (ix == A.nx) {
          const double mfphelp = (capi + sigc) * dist;
          const double ppr = 4.0 / (3.0 * mfphelp + 6.0 * pc_dext);
          res = 1.5 * ppr * sq(X1) / dx3;
        } else {
          const int l = ix + 1;
          const double capl = (double)A.cap[(size_t)(l - 1) * ng + iiig - 1];
          const double dxr = A.xarr[ix + 1] - A.xarr[ix];
          if ((capl + A.sig[l - 1]) * dxr < A.tauddmc) {
            const double mfphelp = (capi + sigc) * dist;
            const double ppr = 4.0 / (3.0 * mfphelp + 6.0 * pc_dext);
            res = 1.5 * ppr * sq(X1) / dx3;
          } else {
            const double mfphelp = (sigc + capi) * dist + (A.sig[l - 1] + capl) * dxr;
            res = 2.0 * sq(X1) / (mfphelp * dx3);
          }
        }
        cright[q - 1] = specig * res * speclump * hr;
      }
      // effective scattering over unlumped groups (:571-584), loop order q
      if (q <= ng - nlump) {
        const int iig = ng + 1 - q;
        const int iiig = glumps[iig - 1];
        const double help = specarr[iiig - 1] * (double)capc[iiig - 1] * capgreyinv;
        cscat[q - 1] = help * denom2;
      }
    }
  }
  // emitgroup within-bin running sums (emitgroup.f:303-320), one thread per bin
  const double* ep = A.emitprob + (size_t)A.nep * (ic - 1);
  for (int iep = threadIdx.x; iep <= A.nep; iep += GB) {
    const int ig0 = iep * A.nepg + 1;
    const int igp1 = min(ig0 + A.nepg - 1, ng);
    double prob = iep == 0 ? 0.0 : ep[iep - 1];
    for (int g = ig0; g <= igp1 - 1; ++g) {
      prob = prob + specarr[g - 1] * (double)capc[g - 1];
      ecum[g - 1] = prob;
    }
  }
  __syncthreads();
  // ---- phase B: running sums
  if (nlump > 0) {
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int q = 0; q < nlump; ++q) { s = s + cdop[q]; cdop[q] = s; }
    } else if (threadIdx.x == 32 && ix > 1) {
      double s = 0.0;
      for (int q = 0; q < nlump; ++q) { s = s + cleft[q]; cleft[q] = s; }
    } else if (threadIdx.x == 64) {
      double s = 0.0;
      for (int q = 0; q < nlump; ++q) { s = s + cright[q]; cright[q] = s; }
    } else if (threadIdx.x == 96) {
      double s = 0.0;
      for (int q = 0; q < ng - nlump; ++q) { s = s + cscat[q]; cscat[q] = s; }
    }
  }
  // ---- phase C: guide tables of the four running sums (see CellTables::guide)
  if (A.T.guide && nlump > 0) {
    __syncthreads();
    const int gm = A.T.guide_m;
    int16_t* gd = A.T.guide + (size_t)(ic - 1) * 4 * (gm + 1);
    for (int t = 0; t < 4; ++t) {
      const double* a = t == 0 ? cdop : (t == 1 ? cleft : (t == 2 ? cright : cscat));
      const int n = t == 3 ? ng - nlump : nlump;
      for (int k = threadIdx.x; k <= gm; k += blockDim.x) {
        const double v = (double)k / (double)gm;  // exact: gm is a power of two
        int lo = 0, hi = (t == 1 && ix == 1) ? 0 : n;  // no left leak from the first shell
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (a[mid] <= v) lo = mid + 1;
          else hi = mid;
        }
        gd[t * (gm + 1) + k] = (int16_t)lo;
      }
    }
  }
}

}  // namespace

int launch_leakage(slg_ctx* ctx, const double* tempinv, const double* sig, const float* cap,
                   const float* capemit, double tauddmc, double taulump, double* opaclump) {
  LeakArgs A{ctx->nx, ctx->ng, ctx->d_xarr, ctx->d_vol, ctx->d_divv, tempinv, sig, ctx->d_wlinv,
             cap, capemit, tauddmc, taulump, opaclump, ctx->nmodel > 1 ? ctx->d_cellmap : nullptr};
  leakage_kernel<float><<<ctx->nx, GB, 0, ctx->stream>>>(A);
  return cuda_check(ctx, cudaGetLastError(), "leakage launch");
}

// leakage_opacity11 on the FP64 opacity (ng, ncell) of the differentiable path.
int launch_leakage64(slg_ctx* ctx, const double* tempinv, const double* sig, const double* cap, double tauddmc,
                     double taulump, double* opaclump) {
  LeakArgsT<double> A{ctx->nx, ctx->ng, ctx->d_xarr, ctx->d_vol, ctx->d_divv, tempinv, sig, ctx->d_wlinv,
                      cap, nullptr, tauddmc, taulump, opaclump, ctx->nmodel > 1 ? ctx->d_cellmap : nullptr};
  leakage_kernel<double><<<ctx->nx, GB, 0, ctx->stream>>>(A);
  return cuda_check(ctx, cudaGetLastError(), "leakage64 launch");
}

// Adjoint of leakage_kernel<double> for opaclump rows 1, 2 (leakage), 7
// (speclump), 8 (caplump) and 11 (doplump): gol (11, ncell) in; adds to gcap
// (ng, ncell) of the cell and its neighbours, gsig and gT.  The lumping masks
// are piecewise constant and contribute nothing.
int launch_leakage64_bwd(slg_ctx* ctx, const double* tempinv, const double* sig, const double* cap,
                         double tauddmc, double taulump, const double* opaclump, const double* gol, double* gcap,
                         double* gsig, double* gT) {
  LeakArgsT<double> A{ctx->nx, ctx->ng, ctx->d_xarr, ctx->d_vol, ctx->d_divv, tempinv, sig, ctx->d_wlinv,
                      cap, nullptr, tauddmc, taulump, const_cast<double*>(opaclump),
                      ctx->nmodel > 1 ? ctx->d_cellmap : nullptr};
  leakage_bwd_kernel<<<ctx->nx, GB, 0, ctx->stream>>>(A, gol, gcap, gsig, gT);
  return cuda_check(ctx, cudaGetLastError(), "leakage adjoint launch");
}

int launch_emitprob(slg_ctx* ctx, const double* tempinv, const float* cap, const double* capgrey,
                    double* emitprob) {
  const size_t shm = sizeof(double) * (ctx->nep > 0 ? ctx->nep : 1);
  emitprob_kernel<<<ctx->nx, 128, shm, ctx->stream>>>(ctx->ng, ctx->nep, ctx->nepg, tempinv, cap, capgrey,
                                                      ctx->d_wlinv, emitprob);
  return cuda_check(ctx, cudaGetLastError(), "emission_probability launch");
}

int build_cell_tables(slg_ctx* ctx, const slg_transport_in* in) {
  const int nx = ctx->nx, ng = ctx->ng;
  const size_t n = (size_t)nx * ng;
  CellTables& T = ctx->tables;
  if (T.nx != nx || T.ng != ng) {
    T.specarr = (double*)scratch(ctx, 12, sizeof(double) * n);
    T.glumps = (int16_t*)scratch(ctx, 13, sizeof(int16_t) * n);
    T.cdf_dop = (double*)scratch(ctx, 14, sizeof(double) * n);
    T.cdf_left = (double*)scratch(ctx, 15, sizeof(double) * n);
    T.cdf_right = (double*)scratch(ctx, 16, sizeof(double) * n);
    T.cdf_scat = (double*)scratch(ctx, 17, sizeof(double) * n);
    T.emitcum = (double*)scratch(ctx, 18, sizeof(double) * n);
    T.nlump = (int32_t*)scratch(ctx, 19, sizeof(int32_t) * nx);
    T.scal = (double*)scratch(ctx, 20, sizeof(double) * SCAL_N * nx);
    // guide entries are int16 positions
    T.guide_m = guide_size(ng);
    T.guide = ng < 32768 ? (int16_t*)scratch(ctx, 72, sizeof(int16_t) * 4 * (T.guide_m + 1) * (size_t)nx) : nullptr;
    if (!T.specarr || !T.glumps || !T.cdf_dop || !T.cdf_left || !T.cdf_right || !T.cdf_scat ||
        !T.emitcum || !T.nlump || !T.scal || (ng < 32768 && !T.guide)) {
      T.nx = T.ng = 0;
      return SLG_ERR_OOM;
    }
    T.nx = nx;
    T.ng = ng;
  }
  TabArgs A;
  A.nx = nx; A.ng = ng; A.nep = ctx->nep; A.nepg = ctx->nepg;
  A.xarr = ctx->d_xarr; A.vxarr = ctx->d_vxarr; A.divv = ctx->d_divv; A.wlinv = ctx->d_wlinv;
  A.tempinv = in->tempinv; A.sig = in->sig; A.capgrey = in->capgrey; A.opaclump = in->opaclump;
  A.emitprob = in->emitprob; A.cap = in->cap; A.tauddmc = in->tauddmc; A.taulump = in->taulump;
  A.T = T;
  A.cellmap = ctx->nmodel > 1 ? ctx->d_cellmap : nullptr;
  cell_tables_kernel<<<nx, GB, 0, ctx->stream>>>(A);
  return cuda_check(ctx, cudaGetLastError(), "cell tables launch");
}

}  // namespace slg

namespace slg {
// Launch of cell_tables_kernel on caller-provided tables and stream (used by
// the entry point that allocates nothing).
int launch_cell_tables_raw(cudaStream_t st, int nx, int ng, int nep, int nepg, const double* xarr,
                           const double* vxarr, const double* divv, const double* wlinv,
                           const slg_transport_in* in, const CellTables& T) {
  TabArgs A;
  A.nx = nx; A.ng = ng; A.nep = nep; A.nepg = nepg;
  A.xarr = xarr; A.vxarr = vxarr; A.divv = divv; A.wlinv = wlinv;
  A.tempinv = in->tempinv; A.sig = in->sig; A.capgrey = in->capgrey; A.opaclump = in->opaclump;
  A.emitprob = in->emitprob; A.cap = in->cap; A.tauddmc = in->tauddmc; A.taulump = in->taulump;
  A.T = T;
  cell_tables_kernel<<<nx, GB, 0, st>>>(A);
  return cudaGetLastError() == cudaSuccess ? SLG_OK : SLG_ERR_CUDA;
}
}  // namespace slg
