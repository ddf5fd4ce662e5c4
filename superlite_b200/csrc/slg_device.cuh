// slg_device.cuh -- device-side constants and helpers shared by the kernels.
//
// Physical constants are those of physconstmod.f:11-51; derived constants are
// written with the Fortran expression order so that the FP64 kernels round
// like the reference (integer powers as explicit products, no FMA contraction:
// the FP64 translation units are compiled with -fmad=false).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace slg {

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
constexpr double pc_amu = 1.66053886e-24;

constexpr double cinv = 1.0 / pc_c;
constexpr double pi_4th = (pc_pi * pc_pi) * (pc_pi * pc_pi);
constexpr double hck = pc_h * pc_c / pc_kb;              // groupmod.f:110
constexpr double ftpi4 = 15.0 / pi_4th;                   // groupmod.f:109
constexpr double ftpi4r = 15.0 / (4.0 * pi_4th);          // groupmod.f:290
constexpr double planck_c1 = 2.0 * pc_h * (pc_c * pc_c);  // physconstmod.f:87
constexpr double planck_c2 = pc_h * pc_c / pc_kb;         // physconstmod.f:88
constexpr double pc_hc = pc_h * pc_c;
constexpr double e2c = pc_e * pc_e;
constexpr double e4c = e2c * e2c;
constexpr double e6c = e4c * e2c;
constexpr double c2c = pc_c * pc_c;
constexpr double c4c = c2c * c2c;
constexpr double cthomson = 8.0 * pc_pi * e4c / (3.0 * (pc_me * pc_me) * c4c);  // physical_opacity.f:51

// ---- exp(x) by Tang's table-driven method (P. T. P. Tang, "Table-driven
// implementation of the exponential function in IEEE floating-point
// arithmetic", ACM TOMS 15 (1989) 144-157), for the opacity build's inner
// loops, whose one exp per line-shell term is their binding work:
//   x = (64 m + j) ln2/64 + r,  |r| <= ln2/128,  exp(x) = 2^m 2^(j/64) e^r,
// with ln2/64 split in a 36-bit head (so that n * head is exact for |n| <
// 2^17) and its remainder, e^r - 1 by its Taylor polynomial of degree 5
// (truncation below 4e-17 relative), 2^(j/64) from a 64-entry table and 2^m
// added to the exponent field.  Arguments outside [-700, 700] go to exp().
// The constants and the table are the output of csrc/exp_table.py.  (A
// 256-entry table with a degree-4 polynomial saves one FMA per exp but was
// slower in the opacity kernels: its shared-memory lookups conflict more.)
constexpr int kExpTabN = 64;
constexpr double kExpInvL = 92.33248261689366;        // 64 / ln 2
constexpr double kExpL1 = 0.010830424696223417;       // ln2/64, 36 significant bits
constexpr double kExpL2 = 2.572804622327669e-14;      // ln2/64 - kExpL1
// 2^(j/64), j = 0..63, correctly rounded
static __constant__ double kExp2Tab[kExpTabN] = {
    1.0, 1.0108892860517005, 1.0218971486541166, 1.0330248790212284,
    1.0442737824274138, 1.0556451783605572, 1.0671404006768237, 1.0787607977571199,
    1.0905077326652577, 1.102382583307841, 1.1143867425958924, 1.1265216186082418,
    1.1387886347566916, 1.1511892299529827, 1.1637248587775775, 1.1763969916502812,
    1.189207115002721, 1.202156731452703, 1.215247359980469, 1.22848053610687,
    1.241857812073484, 1.255380757024691, 1.2690509571917332, 1.2828700160787783,
    1.2968395546510096, 1.3109612115247644, 1.3252366431597413, 1.339667524053303,
    1.3542555469368927, 1.3690024229745905, 1.383909881963832, 1.3989796725383112,
    1.4142135623730951, 1.42961333839197, 1.4451808069770467, 1.460917794180647,
    1.4768261459394993, 1.4929077282912648, 1.5091644275934228, 1.5255981507445384,
    1.5422108254079407, 1.559004400237837, 1.5759808451078865, 1.593142151342267,
    1.6104903319492543, 1.6280274218573478, 1.645755478153965, 1.6636765803267364,
    1.681792830507429, 1.7001063537185235, 1.718619298122478, 1.7373338352737062,
    1.7562521603732995, 1.7753764925265212, 1.7947090750031072, 1.8142521755003989,
    1.8340080864093424, 1.8539791250833855, 1.8741676341103, 1.8945759815869656,
    1.9152065613971474, 1.9360617934922943, 1.9571441241754002, 1.978456026387951,
};

// Copies kExp2Tab into a block's shared array of kExpTabN doubles (call from
// every thread, then __syncthreads()).
__device__ inline void exp_table_load(double* s_tab) {
  for (int k = threadIdx.x; k < kExpTabN; k += blockDim.x) s_tab[k] = kExp2Tab[k];
}

// tab: kExp2Tab in shared memory.  n = nearest integer of x 64/ln2 by the
// add-and-subtract of 1.5 2^52 (|x 64/ln2| < 2^31, so the sum's low 32 bits
// are n in two's complement and the difference is n exactly).  This form
// requires x in [-700, 700] and does not check it: the result's exponent
// field is formed by an integer add, valid for normal results only.
__device__ __forceinline__ double exp_tang_inrange(double x, const double* tab) {
  constexpr double kRound = 6755399441055744.0;  // 1.5 * 2^52
  const double big = fma(x, kExpInvL, kRound);
  const int ni = (int)__double2loint(big);
  const double n = big - kRound;
  double r = fma(-n, kExpL1, x);
  r = fma(-n, kExpL2, r);
  double p = fma(r, 1.0 / 120.0, 1.0 / 24.0);
  p = fma(r, p, 1.0 / 6.0);
  p = fma(r, p, 0.5);
  p = fma(r, p, 1.0);
  p = p * r;  // e^r - 1
  const double s = tab[ni & (kExpTabN - 1)];
  const double v = fma(s, p, s);  // in [0.99, 2): adding m to the exponent field stays normal
  return __hiloint2double(__double2hiint(v) + (ni >> 6) * (1 << 20), __double2loint(v));
}
// Any x: outside [-700, 700], and for NaN, CUDA's exp.
__device__ inline double exp_tang(double x, const double* tab) {
  if (!(fabs(x) <= 700.0)) return exp(x);  // also NaN
  return exp_tang_inrange(x, tab);
}
constexpr double ff_c1a = 4.0 * e6c / (3.0 * pc_h * pc_me * c4c);              // physical_opacity.f:32
constexpr double ff_c1b = pc_pi2 / (3.0 * pc_me * pc_h * pc_c);                 // argument of its sqrt
// Fortran `1.0/3.0` is a real*4 quotient promoted to real*8 as an exponent.
constexpr double third_r4 = (double)(1.0f / 3.0f);

constexpr int FF_NU = 81, FF_NGG = 41;

__host__ __device__ inline double sq(double x) { return x * x; }
__host__ __device__ inline double cube(double x) { return x * x * x; }
__host__ __device__ inline double pow4(double x) { double t = x * x; return t * t; }
__host__ __device__ inline double pow5(double x) { double t = x * x; return t * t * x; }

// MISC/binsrch.f90:3-77.  arr holds n values; returns the 1-based interval
// index (clamped to 1..n-1 unless widerange), -1 for invalid input.
__device__ inline int binsrch(double x, const double* __restrict__ arr, int n, bool widerange) {
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
    const double amin = arr[imin - 1], amid = arr[imid - 1], amax = arr[imax - 1];
    if (x >= amin && x < amid) {
      imax = imid;
      imid = (imax + imin) / 2;
    } else if (x >= amid && x <= amax) {
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
    imid = imid > n - 1 ? n - 1 : imid;
    imid = imid < 1 ? 1 : imid;
  }
  return imid;
}

// groupmod.f:99-120 (specint0); ig is 1-based, wlinv holds grp_wlinv(1:ng+1)
__device__ inline double specint0(double tempinv, const double* __restrict__ wlinv, int ig) {
  double x = hck * tempinv;
  const double dx = x * fabs(wlinv[ig] - wlinv[ig - 1]);
  x = x * 0.5 * (wlinv[ig] + wlinv[ig - 1]);
  if (x >= 300.0) x = 300.0;
  return ftpi4 * dx * cube(x) / (exp(x) - 1.0);
}

// groupmod.f:123-143
__device__ inline double dopspeccalc(double tempinv, const double* __restrict__ wlinv, int ig) {
  double x = hck * tempinv;
  x = x * wlinv[ig];
  if (x >= 300.0) x = 300.0;
  return ftpi4 * pow4(x) / (exp(x) - 1.0);
}

// Integrand of specintv, groupmod.f:263-270
__device__ inline double fplanck(double x) {
  if (x >= 300.0) return 27000000.0 / (exp(300.0) - 1.0);
  return cube(x) / (exp(x) - 1.0);
}
// Integrand of spectintv, groupmod.f:395-402
__device__ inline double fross(double x) {
  if (x >= 300.0) {
    const double e3 = exp(300.0);
    return (8100000000.0 * e3) / sq(e3 - 1.0);
  }
  const double ex = exp(x);
  return (pow4(x) * ex) / sq(ex - 1.0);
}
// One element k (0-based, group offset+k) of specintv mode 0 (groupmod.f:189-198):
// x = hck*tempinv*wlinv, ss = ftpi4*|x2-x1|*f((x1+x2)/2).
__device__ inline double specintv_elem(double hct, const double* __restrict__ wlinv, int g0) {
  const double x1 = hct * wlinv[g0], x2 = hct * wlinv[g0 + 1];
  return ftpi4 * fabs(x2 - x1) * fplanck(0.5 * (x2 + x1));
}
__device__ inline double spectintv_elem(double hct, const double* __restrict__ wlinv, int g0) {
  const double x1 = hct * wlinv[g0], x2 = hct * wlinv[g0 + 1];
  double s = ftpi4r * fabs(x2 - x1) * fross(0.5 * (x2 + x1));
  return s != s ? 0.0 : s;  // groupmod.f:390-392
}

// physconstmod.f:79-93
__device__ inline double planck(double wl, double temp) {
  double b = 1.0 / (wl * temp);
  if (planck_c2 * b >= 300.0) b = 300.0 / planck_c2;
  return planck_c1 * pow5(temp * b) / (exp(planck_c2 * b) - 1.0);
}

// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11).
struct u32x4 { uint32_t a, b, c, d; };
__device__ inline u32x4 philox4x32_10(u32x4 ctr, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    // one 32 x 32 -> 64-bit multiply gives both halves
    const uint64_t p0 = (uint64_t)0xD2511F53u * ctr.a, p1 = (uint64_t)0xCD9E8D57u * ctr.c;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    ctr = u32x4{hi1 ^ ctr.b ^ k0, lo1, hi0 ^ ctr.d ^ k1, lo0};
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return ctr;
}
// The same rounds kept out of line for the event loops, which draw from
// many places: one copy of the rounds instead of one per call site keeps the
// loop within the instruction cache.  Same results as philox4x32_10.
static __device__ __noinline__ u32x4 philox4x32_10_call(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                        uint32_t k0, uint32_t k1) {
  return philox4x32_10(u32x4{c0, c1, c2, c3}, k0, k1);
}
__device__ inline double u52_to_unit(uint32_t w0, uint32_t w1) {
  const uint64_t m = ((uint64_t)w0 << 20) | (w1 >> 12);
  return ((double)m + 0.5) * 0x1p-52;
}

// Per-particle stream: draw k uses counter (k/2, pid, stream), words (0,1) for
// even k and (2,3) for odd k; the odd half is kept for the next draw.
struct PhiloxStream {
  uint32_t k0, k1, pid_lo, pid_hi, stream;
  uint32_t k;
  uint32_t w2, w3;
  __device__ inline void init(uint64_t seed, uint64_t pid, uint32_t s) {
    k0 = (uint32_t)seed; k1 = (uint32_t)(seed >> 32);
    pid_lo = (uint32_t)pid; pid_hi = (uint32_t)(pid >> 32);
    stream = s; k = 0;
  }
  __device__ inline double draw() {
    double r;
    if ((k & 1u) == 0u) {
      const u32x4 o = philox4x32_10_call(k >> 1, pid_lo, pid_hi, stream, k0, k1);
      w2 = o.c; w3 = o.d;
      r = u52_to_unit(o.a, o.b);
    } else {
      r = u52_to_unit(w2, w3);
    }
    ++k;
    return r;
  }
};

__device__ inline uint64_t fnv_mix(uint64_t h, int32_t v) {
  const uint32_t u = (uint32_t)v;
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    h ^= (u >> (8 * b)) & 0xffu;
    h *= 1099511628211ull;
  }
  return h;
}

}  // namespace slg
