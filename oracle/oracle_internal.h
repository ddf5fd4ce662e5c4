// oracle_internal.h -- constants and helpers shared by the oracle's .cpp files.
// TEST INFRASTRUCTURE ONLY (parity checker for the CUDA product).
#ifndef SUPERLITE_ORACLE_INTERNAL_H
#define SUPERLITE_ORACLE_INTERNAL_H
#include <cmath>
#include <cstdint>
#include <vector>
#include "superlite_oracle.h"

namespace orc {

// physconstmod.f:11-51 (values verbatim).  Integer powers are written as
// explicit products; derived constants follow the Fortran expression order.
constexpr double pc_acoef = 7.5657e-15;
constexpr double pc_pi = 3.1415926535897932385;
constexpr double pc_pi2 = 2.0 * pc_pi;
constexpr double pc_pi4 = 4.0 * pc_pi;
constexpr double pc_c = 2.997924562e10;
constexpr double pc_kb = 1.3806505e-16;
constexpr double pc_me = 9.1093826e-28;
constexpr double pc_h = 6.6260693e-27;
constexpr double pc_e = 4.80325e-10;
constexpr double pc_rydberg = 1.0973731534e5;
constexpr double pc_dext = 0.7104;
constexpr double pc_ev = 1.60217653e-12;
constexpr double pc_ang = 1e-8;
constexpr double pc_mbarn = 1e-18;

constexpr double cinv = 1.0 / pc_c;
constexpr double pi_4th = (pc_pi * pc_pi) * (pc_pi * pc_pi);
constexpr double hck = pc_h * pc_c / pc_kb;       // groupmod.f:110
constexpr double ftpi4 = 15.0 / pi_4th;            // groupmod.f:109
constexpr double ftpi4r = 15.0 / (4.0 * pi_4th);   // groupmod.f:290
constexpr double planck_c1 = 2.0 * pc_h * (pc_c * pc_c);  // physconstmod.f:87
constexpr double planck_c2 = pc_h * pc_c / pc_kb;         // physconstmod.f:88
constexpr double pc_hc = pc_h * pc_c;
// physical_opacity.f:32-33 and :51-52
constexpr double e2 = pc_e * pc_e;
constexpr double e4 = e2 * e2;
constexpr double e6 = e4 * e2;
constexpr double c2c = pc_c * pc_c;
constexpr double c4c = c2c * c2c;
constexpr double cthomson = 8.0 * pc_pi * e4 / (3.0 * (pc_me * pc_me) * c4c);
inline double ff_c1() {
  return 4.0 * e6 / (3.0 * pc_h * pc_me * c4c) * std::sqrt(pc_pi2 / (3.0 * pc_me * pc_h * pc_c));
}
// Fortran `1.0/3.0` is a real*4 quotient promoted to real*8 when used as the
// exponent of a real*8 base (diffusion11.f90:336,597; interior_source.f90:258).
constexpr double third_r4 = (double)(1.0f / 3.0f);

inline double sq(double x) { return x * x; }
inline double cube(double x) { return x * x * x; }
inline double pow4(double x) { double t = x * x; return t * t; }
inline double pow5(double x) { double t = x * x; return t * t * x; }

// MISC/binsrch.f90:3-77.  arr holds n values (Fortran arr(1:n)).  Returns the
// 1-based interval index; -1 for invalid input.
inline int binsrch(double x, const double* arr, int n, bool widerange) {
  if (n == 2) {
    int r;
    if (x >= arr[0] && x <= arr[1]) r = 1;
    else if (x < arr[0]) r = 0;
    else if (x > arr[1]) r = n;
    else return -1;
    if (!widerange) r = 1;
    return r;
  }
  int imin = 1, imax = n, imid = (n + 1) / 2;
  while (imax - imin > 1) {
    if (x >= arr[imin - 1] && x < arr[imid - 1]) {
      imax = imid;
      imid = (imax + imin) / 2;
    } else if (x >= arr[imid - 1] && x <= arr[imax - 1]) {
      imin = imid;
      imid = (imax + imin) / 2;
    } else {
      if (x < arr[0]) { imin = 0; imid = 0; break; }
      else if (x > arr[n - 1]) { imin = n; imid = n; break; }
      else return -1;
    }
  }
  if (imid != imin) imid = -1;
  if (!widerange) {
    if (imid > n - 1) imid = n - 1;
    if (imid < 1) imid = 1;
  }
  return imid;
}

// randommod.f:129-170 (mzran of Marsaglia & Zaman), int32 wrap-around.
inline int32_t mzran_next(orc_rnd* s) {
  int32_t imz = (int32_t)((uint32_t)s->part[0] - (uint32_t)s->part[2]);
  if (imz < 0) imz = (int32_t)((uint32_t)imz + 2147483579u);
  s->part[0] = s->part[1];
  s->part[1] = s->part[2];
  s->part[2] = imz;
  s->part[3] = (int32_t)(69069u * (uint32_t)s->part[3] + 1013904243u);
  imz = (int32_t)((uint32_t)imz + (uint32_t)s->part[3]);
  return imz;
}
inline double mzran_real(orc_rnd* s) {
  int32_t imz = mzran_next(s);
  return 0.5 + 0.23283064e-9 * (double)imz;  // randommod.f:169
}

// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11).  Draw k of particle pid
// uses counter (k/2, pid_lo, pid_hi, stream) and key (seed_lo, seed_hi); output
// words (0,1) serve even k and (2,3) odd k.  Two words w0,w1 give the 52-bit
// integer m = w0 2^20 + (w1 >> 12); the draw is (m + 1/2) 2^-52, in (0,1).
inline void philox4x32_10(uint32_t ctr[4], uint32_t key[2]) {
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * ctr[0];
    uint64_t p1 = (uint64_t)0xCD9E8D57u * ctr[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ ctr[1] ^ key[0];
    uint32_t n2 = hi0 ^ ctr[3] ^ key[1];
    ctr[0] = n0; ctr[1] = lo1; ctr[2] = n2; ctr[3] = lo0;
    key[0] += 0x9E3779B9u;
    key[1] += 0xBB67AE85u;
  }
}
inline double philox_real(uint64_t seed, uint64_t pid, uint32_t stream, uint32_t k) {
  uint32_t ctr[4] = {k >> 1, (uint32_t)pid, (uint32_t)(pid >> 32), stream};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  philox4x32_10(ctr, key);
  const int o = (int)(k & 1u) * 2;
  uint64_t m = ((uint64_t)ctr[o] << 20) | (ctr[o + 1] >> 12);
  return ((double)m + 0.5) * 0x1p-52;
}

}  // namespace orc
#endif
