// oracle_eos.cpp -- CPU restatement of the LTE equation of state.
//
// TEST INFRASTRUCTURE ONLY (see superlite_oracle.h).
//
// ionsmod.f:160-356 (ions_solve_eos with its contained saha_nelec) and
// GAS/eos_update.f:20-45 (ground-state occupation densities).  The reference
// evaluates the partition functions only while they are all zero
// (ionsmod.f:209), i.e. once, at the temperature of the first cell of the
// first call, and reuses them for every later cell and step; orc_partition
// gives those values for a chosen temperature and orc_saha_eos takes them as
// input.
#include <cmath>
#include <limits>
#include <vector>
#include "oracle_internal.h"
#include "superlite_oracle.h"

using namespace orc;

namespace {

struct Saha {
  const orc_ion* ion;
  double kti, sahac2;
  std::vector<double> n;   // (nstage_all, nelem): stage populations of the last saha_nelec
  std::vector<double> ne;  // (nelem)
};

// saha_nelec, ionsmod.f:298-354.  Returns 0 or -1 when a normalisation sum is
// invalid (the reference stops).
int saha_nelec(Saha& s, const double* natomfr, double* nelec_out) {
  const orc_ion* I = s.ion;
  const int ns = I->nstage;
  for (int iz = 0; iz < I->nelem; ++iz) {
    const int nion = I->ni[iz];
    double* n = &s.n[(size_t)iz * ns];
    const double* e = I->e + (size_t)iz * ns;
    const double* q = I->q + (size_t)iz * ns;
    double help = 0.0;
    // recursively n_(i+1) from an arbitrary n at istart (restart higher on overflow)
    for (int istart = 1; istart <= nion - 1; ++istart) {
      n[istart - 1] = 1.0;
      for (int ii = istart + 1; ii <= nion; ++ii) {
        help = s.sahac2 * std::exp(-s.kti * e[ii - 2]) * n[ii - 2] * q[ii - 1] / q[ii - 2];
        n[ii - 1] = help;
      }
      if (help < std::numeric_limits<double>::max()) break;
    }
    double nsum = 0.0;
    for (int ii = 0; ii < nion; ++ii) nsum = nsum + n[ii];
    if (nsum != nsum || nsum > std::numeric_limits<double>::max() || nsum < std::numeric_limits<double>::min())
      return -1;
    nsum = 1.0 / nsum;
    for (int ii = 0; ii < nion; ++ii) n[ii] = n[ii] * nsum;
    double z = 0.0;
    for (int ii = 2; ii <= nion; ++ii) z = z + (double)(ii - 1) * n[ii - 1];
    s.ne[iz] = z;
  }
  double nel = 0.0;
  for (int iz = 0; iz < I->nelem; ++iz) nel = nel + natomfr[iz + 1] * s.ne[iz];
  *nelec_out = nel;
  return 0;
}

}  // namespace

extern "C" {

void orc_partition(int nelem, int nstage, int nlev, const int32_t* ni, const int32_t* nlevel,
                   const double* glev, const double* elev, double temp, double* q) {
  const double kti = 1.0 / (pc_kb * temp);
  for (int iz = 0; iz < nelem; ++iz) {
    for (int ii = 0; ii < nstage; ++ii) q[(size_t)iz * nstage + ii] = 0.0;
    for (int ii = 0; ii < ni[iz] - 1; ++ii) {
      const size_t o = ((size_t)iz * nstage + ii) * nlev;
      double s = 0.0;
      for (int k = 0; k < nlevel[(size_t)iz * nstage + ii]; ++k) s = s + glev[o + k] * std::exp(-kti * elev[o + k]);
      q[(size_t)iz * nstage + ii] = s;
    }
    q[(size_t)iz * nstage + ni[iz] - 1] = 1.0;
  }
}

int orc_saha_eos(const orc_ion* ion, int ncell, const double* temp, const double* natom, const double* vol,
                 const double* natomfr, double acc, double* nelec, int32_t noc, double* oc, double* ginv,
                 int32_t* iconv_out) {
  const int nconv = 40;
  const int ns = ion->nstage;
  Saha s;
  s.ion = ion;
  s.n.assign((size_t)ion->nelem * ns, 0.0);
  s.ne.assign(ion->nelem, 0.0);
  for (int i = 0; i < ncell; ++i) {
    const double* fr = natomfr + (size_t)i * (ion->nelem + 1);
    const double ndens = natom[i] / vol[i];
    const double T = temp[i];
    s.kti = 1.0 / (pc_kb * T);
    const double sahac = std::pow(pc_pi2 * pc_me * pc_kb * T / (pc_h * pc_h), 1.5);
    double nel = nelec[i];
    double nec_nel[2] = {0.0, 0.0};
    double nec_err[2] = {1e10, -1e10};
    int iprev = 0;
    int iconv;
    for (iconv = 1; iconv <= nconv; ++iconv) {
      s.sahac2 = 2.0 / (nel * ndens) * sahac;
      double nel_new = 0.0;
      if (saha_nelec(s, fr, &nel_new)) return -(i + 1);
      const double err = nel / nel_new - 1.0;
      if (std::fabs(err) < acc) {
        if (iconv > 1) nel = nel_new;
        break;
      }
      // replace the saved value on the same side of zero (maxloc of err*nec%err)
      const int ih = (err * nec_err[1] > err * nec_err[0]) ? 1 : 0;
      nec_nel[ih] = nel;
      nec_err[ih] = err;
      if (iconv == 1) {
        nel = 1.5 * nel_new - 0.5 * nel;
        nel = std::min(3.0 * nel_new, nel);
        nel = std::max(0.33 * nel_new, nel);
      } else {
        const int ib = (std::fabs(nec_err[1]) > std::fabs(nec_err[0])) ? 1 : 0;
        const double help = std::fabs(nec_err[0] / nec_err[1]);
        double ynew;
        if ((ib + 1) != iprev && help < 1e5 && help > 1e-5) ynew = 0.0;
        else ynew = 0.001 * nec_err[ib];
        iprev = ib + 1;
        const double dxdy = (nec_nel[1] - nec_nel[0]) / (nec_err[1] - nec_err[0]);
        nel = nec_nel[0] - dxdy * (nec_err[0] - ynew);
        if (nel <= 0.0) return -(i + 1);
      }
    }
    nelec[i] = nel;
    if (iconv_out) iconv_out[i] = iconv;
    // eos_update.f:37-45 for the first noc stages of every element
    for (int iz = 0; iz < ion->nelem; ++iz) {
      for (int ii = 0; ii < noc; ++ii) {
        const size_t o = (size_t)i + (size_t)ncell * ((size_t)ii + (size_t)noc * iz);
        if (ii < ion->ni[iz]) {
          const size_t k = (size_t)iz * ns + ii;
          ginv[o] = 1.0 / ion->g1[k];
          oc[o] = natom[i] * fr[iz + 1] * ion->g1[k] * s.n[k] / (ion->q[k] * vol[i]);
        } else {
          ginv[o] = 1.0;
          oc[o] = 0.0;
        }
      }
    }
  }
  return 0;
}

}  // extern "C"
