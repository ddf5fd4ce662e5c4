// oracle_grid.cpp -- DDMC leakage opacities, emission probabilities and group
// sampling of the reference, restated on the CPU.
// TEST INFRASTRUCTURE ONLY (parity checker for the CUDA product).
//
// GRID/leakage_opacity11.f90:3-174, GRID/emission_probability.f90:3-67,
// GRID/emitgroup.f:3-54.  1-D spherical grid without void cells:
// grd_icell(ix,1,1) = ix.
#include "oracle_internal.h"

using namespace orc;

extern "C" {

void orc_leakage_opacity11(int nx, int ng, const double* xarr, const double* vol,
                           const double* divv, const double* tempinv, const double* sig,
                           const float* cap, const float* capemit, const double* wlinv,
                           double tauddmc, double taulump, double* opaclump) {
  auto X = [&](int i) { return xarr[i - 1]; };
  auto dx = [&](int i) { return xarr[i] - xarr[i - 1]; };
  auto CAP = [&](int ig, int l) { return (double)cap[(size_t)(ig - 1) + (size_t)ng * (l - 1)]; };
  auto CEM = [&](int ig, int l) {
    return capemit ? (double)capemit[(size_t)(ig - 1) + (size_t)ng * (l - 1)] : 0.0;
  };
  std::vector<double> specarr(ng);
  for (int i = 1; i <= nx; ++i) {
    const int l = i;
    double* ol = opaclump + (size_t)11 * (l - 1);
    for (int k = 0; k < 11; ++k) ol[k] = 0.0;
    const int icnb1 = i - 1 > 1 ? i - 1 : 1;
    const int icnb2 = i + 1 < nx ? i + 1 : nx;
    const double dist = dx(i);
    orc_specintv(tempinv[l - 1], wlinv, ng, ng, 1, 0, specarr.data());
    auto lumpable = [&](int ig) {
      return CAP(ig, l) * dist >= taulump && (sig[l - 1] + CAP(ig, l)) * dist >= tauddmc;
    };
    double speclump = 0.0;
    for (int ig = 1; ig <= ng; ++ig)
      if (lumpable(ig)) speclump = speclump + specarr[ig - 1];
    speclump = speclump > 0.0 ? 1.0 / speclump : 0.0;
    ol[6] = speclump;
    double caplump = 0.0, capemitlump = 0.0, emitmax = 0.0;
    int igemitmax = 0;
    for (int ig = 1; ig <= ng; ++ig) {
      if (CAP(ig, l) * dist < taulump) continue;
      if ((sig[l - 1] + CAP(ig, l)) * dist < tauddmc) continue;
      double help = specarr[ig - 1] * CAP(ig, l);
      caplump = caplump + help;
      if (help > emitmax) { emitmax = help; igemitmax = ig; }
    }
    for (int ig = 1; ig <= ng; ++ig) {
      if (CAP(ig, l) * dist < taulump) continue;
      if ((sig[l - 1] + CAP(ig, l)) * dist < tauddmc) continue;
      double help = specarr[ig - 1] * CEM(ig, l);
      capemitlump = capemitlump + help;
      if (help > emitmax) { emitmax = help; igemitmax = ig; }
    }
    double doplump = 0.0;
    if (divv[l - 1] >= 0.0) {
      for (int ig = 1; ig <= ng - 1; ++ig) {
        if (CAP(ig, l) * dist < taulump) continue;
        if (CAP(ig + 1, l) * dist >= taulump) continue;
        if ((sig[l - 1] + CAP(ig, l)) * dist < tauddmc) continue;
        double help = orc_dopspeccalc(tempinv[l - 1], wlinv, ig) * divv[l - 1] / (3.0 * pc_c);
        doplump = doplump + help;
      }
    } else {
      for (int ig = ng; ig >= 2; --ig) {
        if (CAP(ig, l) * dist < taulump) continue;
        if (CAP(ig - 1, l) * dist >= taulump) continue;
        if ((sig[l - 1] + CAP(ig, l)) * dist < tauddmc) continue;
        double help = orc_dopspeccalc(tempinv[l - 1], wlinv, ig - 1) * divv[l - 1] / (3.0 * pc_c);
        doplump = doplump - help;
      }
    }
    ol[7] = caplump;
    ol[8] = capemitlump;
    ol[9] = (double)igemitmax;
    ol[10] = doplump;
    const double vterm = 3.0 * vol[l - 1] / pc_pi4;
    for (int ig = 1; ig <= ng; ++ig) {
      if (CAP(ig, l) * dist < taulump) continue;
      if ((sig[l - 1] + CAP(ig, l)) * dist < tauddmc) continue;
      double specval = specarr[ig - 1];
      bool lhelp;
      if (i == 1) lhelp = true;
      else lhelp = (CAP(ig, icnb1) + sig[icnb1 - 1]) * dx(i - 1) < tauddmc;
      if (lhelp) {
        double help = (CAP(ig, l) + sig[l - 1]) * dx(i);
        double ppl = 4.0 / (3.0 * help + 6.0 * pc_dext);
        ol[0] = ol[0] + (specval * speclump) * 1.5 * ppl * sq(X(i)) / vterm;
      } else {
        double help = (sig[l - 1] + CAP(ig, l)) * dx(i) + (sig[icnb1 - 1] + CAP(ig, icnb1)) * dx(i - 1);
        ol[0] = ol[0] + (specval * speclump) * 2.0 * sq(X(i)) / (help * 3.0 * vol[l - 1] / pc_pi4);
      }
      if (i == nx) lhelp = true;
      else lhelp = (CAP(ig, icnb2) + sig[icnb2 - 1]) * dx(i + 1) < tauddmc;
      if (lhelp) {
        double help = (CAP(ig, l) + sig[l - 1]) * dx(i);
        double ppr = 4.0 / (3.0 * help + 6.0 * pc_dext);
        ol[1] = ol[1] + (specval * speclump) * 1.5 * ppr * sq(X(i + 1)) / vterm;
      } else {
        double help = (sig[l - 1] + CAP(ig, l)) * dx(i) + (sig[icnb2 - 1] + CAP(ig, icnb2)) * dx(i + 1);
        ol[1] = ol[1] + (specval * speclump) * 2.0 * sq(X(i + 1)) / (help * 3.0 * vol[l - 1] / pc_pi4);
      }
    }
  }
}

// GRID/emission_probability.f90:40-63 (LTE)
void orc_emission_probability(int nx, int ng, int nep, int nepg, const double* tempinv,
                              const float* cap, const double* capgrey, const double* wlinv,
                              double* emitprob) {
  if (ng == 1) {
    for (int l = 0; l < nx; ++l) emitprob[(size_t)nep * l] = capgrey[l];
    return;
  }
  std::vector<double> specarr(ng);
  for (int l = 1; l <= nx; ++l) {
    orc_specintv(tempinv[l - 1], wlinv, ng, ng, 1, 0, specarr.data());
    int ig = 1;
    double help = 0.0;
    for (int iep = 1; iep <= nep - 1; ++iep) {
      int top = iep * nepg < ng ? iep * nepg : ng;
      int nepg_ = top - ig + 1;
      int igp1 = ig + nepg_ - 1;
      double s = 0.0;
      for (int g = ig; g <= igp1; ++g)
        s = s + specarr[g - 1] * (double)cap[(size_t)(g - 1) + (size_t)ng * (l - 1)];
      help = help + s;
      emitprob[(size_t)(iep - 1) + (size_t)nep * (l - 1)] = help;
      ig = igp1 + 1;
    }
    emitprob[(size_t)(nep - 1) + (size_t)nep * (l - 1)] = capgrey[l - 1];
  }
}

// GRID/emitgroup.f:3-54 (LTE).  ic is 1-based; returns the 1-based group.
int orc_emitgroup(double r, int ic, int ng, int nep, int nepg, const double* tempinv,
                  const float* cap, const double* capgrey, const double* emitprob,
                  const double* wlinv) {
  const double* ep = emitprob + (size_t)nep * (ic - 1);
  double r1 = r * capgrey[ic - 1];
  int iep = orc::binsrch(r1, ep, nep, true);
  if (iep < 0) iep = 0;  // invalid search (NaN): the reference indexes out of bounds here
  int ig = iep * nepg + 1;
  int igp1 = ig + nepg - 1 < ng ? ig + nepg - 1 : ng;
  int nepg_ = igp1 - ig + 1;
  std::vector<double> specval(nepg_ > 0 ? nepg_ : 1);
  if (nepg_ > 0) orc_specintv(tempinv[ic - 1], wlinv, ng, nepg_, ig, 0, specval.data());
  double prob = iep == 0 ? 0.0 : ep[iep - 1];
  int l = 0;
  const int ig0 = ig;
  if (ig0 > igp1 - 1) return ig0;  // zero-trip DO loop leaves the start value
  for (ig = ig0; ig <= igp1 - 1; ++ig) {
    l = l + 1;
    prob = prob + specval[l - 1] * (double)cap[(size_t)(ig - 1) + (size_t)ng * (ic - 1)];
    if (prob > r1) return ig;
  }
  return igp1;
}

}  // extern "C"
