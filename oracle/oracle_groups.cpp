// oracle_groups.cpp -- Planck group integrals, binary search and RNGs of the
// reference, restated on the CPU.  TEST INFRASTRUCTURE ONLY (parity checker).
//
// groupmod.f:99-404 (specint0, dopspeccalc, specintv, spectintv),
// physconstmod.f:79-93 (planck), MISC/binsrch.f90:3-77, randommod.f:25-116.
#include "oracle_internal.h"

using namespace orc;

extern "C" {

// groupmod.f:99-120
double orc_specint0(double tempinv, const double* wlinv, int ig) {
  double x = hck * tempinv;
  double dx = x * std::fabs(wlinv[ig] - wlinv[ig - 1]);
  x = x * 0.5 * (wlinv[ig] + wlinv[ig - 1]);
  if (x >= 300.0) x = 300.0;
  return ftpi4 * dx * cube(x) / (std::exp(x) - 1.0);
}

// groupmod.f:123-143
double orc_dopspeccalc(double tempinv, const double* wlinv, int ig) {
  double x = hck * tempinv;
  x = x * wlinv[ig];  // grp_wlinv(ig+1)
  if (x >= 300.0) x = 300.0;
  return ftpi4 * pow4(x) / (std::exp(x) - 1.0);
}

}  // extern "C"

namespace {
inline double fplanck(double x) {  // groupmod.f:263-270
  if (x >= 300.0) return 27000000.0 / (std::exp(300.0) - 1.0);
  return cube(x) / (std::exp(x) - 1.0);
}
inline double fross(double x) {  // groupmod.f:395-402
  if (x >= 300.0) {
    double e3 = std::exp(300.0);
    return (8100000000.0 * e3) / sq(e3 - 1.0);
  }
  double ex = std::exp(x);
  return (pow4(x) * ex) / sq(ex - 1.0);
}

template <class F>
void newton_cotes(double tempinv, const double* wlinv, int ng, int n, int offset,
                         int mode, double* ss, double norm, F f, bool nan_to_zero) {
  // groupmod.f:146-272 and :275-404 share this body (different f and norm).
  if (offset + n > ng + 1) {
    for (int k = 0; k < n; ++k) ss[k] = -1.0;
    return;
  }
  std::vector<double> x(n + 1);
  const double hct = hck * tempinv;
  for (int k = 0; k <= n; ++k) x[k] = hct * wlinv[offset - 1 + k];
  switch (mode) {
    case 0:
      for (int k = 0; k < n; ++k)
        ss[k] = norm * std::fabs(x[k + 1] - x[k]) * f(0.5 * (x[k + 1] + x[k]));
      break;
    case 1: {
      const double onehalf = norm / 2.0;
      for (int k = 0; k < n; ++k)
        ss[k] = onehalf * std::fabs(x[k + 1] - x[k]) * (f(x[k + 1]) + f(x[k]));
      break;
    }
    case 2: {
      const double one6th = norm / 6.0;
      for (int k = 0; k < n; ++k)
        ss[k] = one6th * std::fabs(x[k + 1] - x[k]) *
                (f(x[k + 1]) + f(x[k]) + 4.0 * f(0.5 * (x[k + 1] + x[k])));
      break;
    }
    case 11: {
      const double one90th = norm / 90.0;
      for (int k = 0; k < n; ++k) {
        double f2 = 12.0 * f(0.5 * (x[k + 1] + x[k])) +
                    32.0 * (f(0.25 * x[k + 1] + 0.75 * x[k]) + f(0.75 * x[k + 1] + 0.25 * x[k]));
        ss[k] = one90th * std::fabs(x[k + 1] - x[k]) * (7.0 * (f(x[k + 1]) + f(x[k])) + f2);
      }
      break;
    }
    default:
      for (int k = 0; k < n; ++k) ss[k] = -1.0;
  }
  if (nan_to_zero)
    for (int k = 0; k < n; ++k)
      if (ss[k] != ss[k]) ss[k] = 0.0;
}

}  // namespace

extern "C" {

void orc_specintv(double tempinv, const double* wlinv, int ng, int n, int offset, int mode,
                  double* ss) {
  newton_cotes(tempinv, wlinv, ng, n, offset, mode, ss, ftpi4, fplanck, false);
}

void orc_spectintv(double tempinv, const double* wlinv, int ng, int n, int offset, int mode,
                   double* ss) {
  newton_cotes(tempinv, wlinv, ng, n, offset, mode, ss, ftpi4r, fross, true);
}

// physconstmod.f:79-93
double orc_planck(double wl, double temp) {
  double b = 1.0 / (wl * temp);
  if (planck_c2 * b >= 300.0) b = 300.0 / planck_c2;
  return planck_c1 * pow5(temp * b) / (std::exp(planck_c2 * b) - 1.0);
}

// MISC/binsrch.f90:3-77 (arr is 1-based in the comments, 0-based here).
int orc_binsrch(double x, const double* arr, int n, int widerange) {
  return orc::binsrch(x, arr, n, widerange != 0);
}

// randommod.f:103-126
void orc_rnd_init(int n, int ioffset, orc_rnd* states) {
  orc_rnd st;
  st.part[0] = 521288629;
  st.part[1] = 362436069;
  st.part[2] = 16163801;
  st.part[3] = 1131199299;
  int64_t nadv = (int64_t)n * ioffset * 4;
  for (int64_t i = 0; i < nadv; ++i) orc::mzran_next(&st);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < 4; ++j) states[i].part[j] = orc::mzran_next(&st);
}

double orc_rnd_r(orc_rnd* s) { return orc::mzran_real(s); }

double orc_philox_draw(uint64_t seed, uint64_t pid, uint32_t stream, uint32_t k) {
  return orc::philox_real(seed, pid, stream, k);
}

}  // extern "C"
