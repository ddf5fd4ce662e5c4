// transport_mixed.cu -- mixed-precision form of the IMC/DDMC particle loop.
//
// Same algorithm and event logic as transport_impl.cuh (particle_advance.f90,
// transport11.f90, diffusion11.f90), with a split of precisions:
//   FP64: particle position x (shell-radius comparisons and the distance to a
//         shell boundary), energy weights e/e0, and the tally accumulation
//         (Kahan-compensated register sums flushed with FP64 atomics);
//   FP32: free-flight distances, Doppler distance, direction cosine mu, fluid
//         velocity, wavelength, DDMC event time and leak probabilities, with
//         fast single-precision log/exp, and 23-bit random numbers (one
//         Philox4x32-10 block of four per event, stream 2 of the particle).
// Cell factors whose magnitude leaves the FP32 range are formed in FP64 and
// rounded once: shell volume factors (x_b^3 - x_a^3 reaches 1e43 cm^3 at a
// few days, above FLT_MAX), Planck group fractions deep in the Wien tail,
// and 1/capgrey.  The DDMC branch is
// picked by comparing r * (sum of rates) against running sums of the rates,
// with the effective-scatter rate exactly zero when every group is lumped
// (its FP64 value, (1 - emitlump) caplump, is rounding noise of a sum that is
// one by construction), so single-precision rounding cannot select the
// impossible scatter branch.
// Results agree with the FP64 form statistically, not event by event.
// Compiled with FMA contraction enabled.
#include <cuda_runtime.h>
#include <cfloat>
#include "slg_device.cuh"
#include "slg_internal.h"
#include "transport_impl.cuh"

namespace slg {
namespace {

constexpr int MIX_BLOCK = 128;
constexpr float cinvf = (float)cinv;
constexpr float pc_cf = (float)pc_c;
constexpr float dextf = (float)pc_dext;

// One Philox4x32-10 block, kept out of line: draw() is called from about
// twenty places of the event code, and one shared copy of the rounds keeps
// the loop small enough for the instruction cache (measured: with the copies
// inlined, "no instruction" was the largest warp stall).
__device__ __noinline__ u32x4 philox_block(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                           uint32_t k1) {
  return philox4x32_10(u32x4{c0, c1, c2, c3}, k0, k1);
}

// Per-particle stream of 23-bit uniforms, (m + 1/2) 2^-23 in (0,1).  Event n
// of the particle draws from Philox blocks with counter word 0 = 4 n + b
// (b = 0, 1, 2, 3 for its 1st-4th, 5th-8th ... draw: room for 16 draws; an
// event here draws at most 7), words 1-2 = the particle, word 3 = the stream.  Block 0 of every event is made at the top of the
// event loop, where the warp's lanes are converged: one Philox call per
// iteration for the whole warp, instead of a call wherever some lane's buffer
// ran out (with lanes out of step, that was every draw site, with a quarter
// of the lanes active).
struct PhiloxStream32 {
  uint32_t k0, k1, pid_lo, pid_hi, stream;
  uint32_t ev, j;  // event number, draws taken in this event
  uint32_t w[4];
  __device__ inline void init(uint64_t seed, uint64_t pid, uint32_t s) {
    k0 = (uint32_t)seed; k1 = (uint32_t)(seed >> 32);
    pid_lo = (uint32_t)pid; pid_hi = (uint32_t)(pid >> 32);
    stream = s;
    ev = 0;
    j = 0;
  }
  __device__ inline void begin_event(uint32_t n) {
    ev = n;
    j = 0;
    const u32x4 o = philox_block(n << 2, pid_lo, pid_hi, stream, k0, k1);
    w[0] = o.a; w[1] = o.b; w[2] = o.c; w[3] = o.d;
  }
  __device__ inline float draw() {
    const uint32_t i = j & 3u;
    if (i == 0u && j != 0u) {  // a 5th, 9th ... draw in one event (rare)
      const u32x4 o = philox_block((ev << 2) | (j >> 2), pid_lo, pid_hi, stream, k0, k1);
      w[0] = o.a; w[1] = o.b; w[2] = o.c; w[3] = o.d;
    }
    ++j;
    const uint32_t u = i == 0u ? w[0] : (i == 1u ? w[1] : (i == 2u ? w[2] : w[3]));
    // (m + 1/2) 2^-23 for the top 23 bits m: 1 + m 2^-23 (the bits under the
    // exponent of 1) minus 1 - 2^-24, exact (both operands in [1/2, 2])
    return __uint_as_float(0x3F800000u | (u >> 9)) - 0.99999994f;
  }
};

struct PtclM {
  double x, e, e0;
  float mu, wl, vx;
  int ix, ig, itype, stat, idist;
};

__device__ inline void kahan_add(double& s, double& c, double v) {
  const double y = v - c;
  const double t = s + y;
  c = (t - s) - y;
  s = t;
}

// relativistic aberration of a direction cosine, (mu + b) / (1 + b mu), kept
// in [-1, 1]: single-precision rounding can leave |mu| a few ulp above 1,
// which makes the chord through the centre (1 - mu^2 < 0) undefined
__device__ inline float aberrate(float mu, float b) {
  const float m = (mu + b) / (1.0f + b * mu);
  return fminf(fmaxf(m, -1.0f), 1.0f);
}

// opacity of group ig in cell ic (1-based over all models' cells)
__device__ inline float capf(const TrnArgs& A, int ig, int ic) {
  return __ldg(A.cap + (size_t)(ic - 1) * A.ng + (ig - 1));
}

// Sentinels of the rate table's first component (a rate is >= 0).
constexpr float kRateLumped = -1.0f;  // cap * dist >= taulump in a shell with lumped groups
constexpr float kRateIMC = -2.0f;     // (sig + cap) * dist < tauddmc: IMC in this shell

// emitgroup (emitgroup.f:3-54) as a search of the shell's emission CDF
// (running sums of specint0 * cap over the groups, divided by capgrey) through
// its guide table: the group with the same probability w_g cap_g / capgrey,
// from one guide load and one round of loads; 1-based.
__device__ inline int emitgroup_mix(const TrnArgs& A, int gc, float r) {
  const float* a = A.emit32 + (size_t)gc * A.ng;
  const int16_t* g = A.eguide + (size_t)gc * (A.T.guide_m + 1);
  const int k = (int)(r * (float)A.T.guide_m);  // exact: guide_m is a power of two and r < 1
  return 1 + first_gt_range32(a, g[k], g[k + 1], A.ng, r);
}

// one IMC event (transport11.f90) in mixed precision
__device__ inline void transport11_mix(const TrnArgs& A, const MView& v, PtclM& p, PhiloxStream32& rng,
                                       double& eraddens,
                                       double& totevelo, int& ierr) {
  int& ix = p.ix;
  int& ig = p.ig;
  float& mu = p.mu;
  float& wl = p.wl;
  float& vx = p.vx;
  const int ic = ix;
  const int gc = v.co + ic - 1;  // 0-based index of the cell over all models
  const MixCell& R = A.mcell[gc];  // this shell's record (one line), read where needed
  ierr = 0;
  eraddens = 0.0;
  float elabfact = 1.0f - mu * vx * cinvf;
  const float elabfactold = elabfact;
  const float far = R.far;
  const double Xa = R.xa, Xb = R.xb;
  const double x = p.x, mud = (double)mu;
  double dbd;
  int ixnext;
  // The radicands are >= 0 in exact arithmetic (x <= Xb; the inner branch is
  // taken only when the chord meets the inner shell).  This unit contracts to
  // FMA, and Xb*Xb - round(x*x) with x == Xb is the (signed) rounding error of
  // the square: a particle on its outer edge with |mu| < ~1e-8 would get a
  // NaN distance, so the radicands are clamped at 0.
  // outward unless the chord meets the inner shell: mu >= -sqrt(1 - (Xa/x)^2)
  // (transport11.f90:95-103) without its FP64 division and square root
  if (ix == 1 || mud >= 0.0 || sq(mud) * sq(x) <= sq(x) - sq(Xa)) {
    dbd = fabs(sqrt(fmax(sq(Xb) - (1.0 - sq(mud)) * sq(x), 0.0)) - mud * x);
    ixnext = ix + 1;
  } else {
    dbd = fabs(sqrt(fmax(sq(Xa) - (1.0 - sq(mud)) * sq(x), 0.0)) + mud * x);
    ixnext = ix - 1;
  }
  if (dbd != dbd) { ierr = 1; return; }
  const float db = (float)dbd;
  const float sigc = R.sig;
  float dthm, dcol, ddop;
  if (sigc > 0.f) dthm = __fdividef(-__logf(rng.draw()), elabfact * sigc);
  else dthm = far;
  const float capc = capf(A, ig, gc + 1);
  if (capc <= 0.f) dcol = far;
  else dcol = __fdividef(-__logf(rng.draw()), elabfact * capc);
  const float dvdr = R.dvdr;
  if (dvdr > 0.f && ig < A.ng) ddop = __fdividef(3.0f * pc_cf, R.divv) * (elabfact - wl * (float)A.wlinv[ig]);
  else if (dvdr < 0.f && ig > 1) ddop = __fdividef(3.0f * pc_cf, R.divv) * (elabfact - wl * (float)A.wlinv[ig - 1]);
  else ddop = far;
  if (ddop < 0.f) ddop = far;
  float d = dcol;
  int im = 1;
  if (dthm < d) { d = dthm; im = 2; }
  if (ddop < d) { d = ddop; im = 3; }
  if (db < d) { d = db; im = 4; }
  p.idist = im;
  if (dcol != dcol || dthm != dthm || ddop != ddop) { ierr = 3; return; }
  if (d < 0.f) { ierr = 4; return; }
  // position in FP64; an event at the boundary lands exactly on the shell edge
  // event kind with the reference's precedence (transport11.f90:256-489)
  const bool is_thm = d == dthm, is_col = !is_thm && d == dcol;
  const bool is_b = !is_thm && !is_col && d == db;
  // An FP32 event distance may round past the FP64 boundary distance (d <=
  // (float)dbd but d > dbd); the event then happens on the shell edge, and
  // the FP64 position stays inside [Xa, Xb] so that the next boundary
  // distance is defined (a position past Xb with |mu| small gives a NaN).
  const double dd = is_b ? dbd : fmin((double)d, dbd);
  double xnew = sqrt(fmax(sq(x) + sq(dd) + 2.0 * dd * x * mud, 0.0));  // (x + dd mu)^2 + dd^2 (1 - mu^2)
  if (!is_b) xnew = fmin(fmax(xnew, Xa), Xb);
  p.x = xnew;
  // FP32 quotients of FP64-formed terms (no FP64 division on the event path)
  vx = __fdividef((float)(R.vxa * (Xb - xnew) + R.vxb * (xnew - Xa)), R.dist);
  mu = xnew == 0.0 ? 1.0f : fminf(fmaxf(__fdividef((float)(x * mud + dd), (float)xnew), -1.0f), 1.0f);
  eraddens = p.e * (double)(elabfact * elabfact) * dd * cinv;
  elabfact = 1.0f - mu * vx * cinvf;
  if (xnew < R.x0) {
    p.x = R.x0;
    vx = (float)A.vxarr[v.xo];
    ix = 1;
    mu = 1.0f - rng.draw();
    return;
  }
  double help;
  if (is_thm || is_col) {
    const float r1 = rng.draw();
    mu = 1.0f - 2.0f * r1;
    mu = aberrate(mu, vx * cinvf);
  } else if (is_b) {
    if ((mu >= 0.f && ix == v.nx) || ixnext > v.nx) { p.stat = 1; return; }
  }
  if (is_thm) {
    const float f = 1.0f - mu * vx * cinvf;
    wl = __fdividef(wl * f, elabfact);
    help = (double)__fdividef(elabfact, f);
    totevelo = totevelo + p.e * (1.0 - help);
    p.e = p.e * help;
    p.e0 = p.e0 * help;
  } else if (is_col) {
    rng.draw();  // the reference's unused draw (transport11.f90:313)
    const float f = 1.0f - mu * vx * cinvf;
    help = (double)__fdividef(elabfact, f);
    totevelo = totevelo + p.e * (1.0 - help);
    p.e = p.e * help;
    p.e0 = p.e0 * help;
    if (A.ng != 1) {
      ig = emitgroup_mix(A, gc, rng.draw());
      if (((sigc + capf(A, ig, gc + 1)) * R.dist >= (float)A.tauddmc) && !A.puretran) p.itype = 2;
    }
    if (p.itype == 2) {
      const double g = (double)(vx * mu * cinvf);
      totevelo = totevelo + p.e * g;
      p.e = p.e * (1.0 - g);
      p.e0 = p.e0 * (1.0 - g);
    } else {
      const float r1 = rng.draw();
      wl = 1.0f / ((1.0f - r1) * (float)A.wlinv[ig - 1] + r1 * (float)A.wlinv[ig]);
      wl = wl * (1.0f - vx * mu * cinvf);
    }
  } else if (is_b) {
    const bool out = ixnext > ix;
    const int l = out ? ix + 1 : ix - 1;
    const float capl = capf(A, ig, v.co + l), sigl = out ? R.sigr : R.sigl;
    const float dxl = out ? R.dxr : R.dxl;
    const double edge = out ? Xb : Xa;
    if ((sigl + capl) * dxl < (float)A.tauddmc || A.puretran) {
      p.x = edge;
      vx = (float)(out ? R.vxb : R.vxa);
      ix = l;
    } else {
      mu = aberrate(mu, -vx * cinvf);
      float hp = (capl + sigl) * dxl;
      hp = __fdividef(4.0f, 3.0f * hp + 6.0f * dextf);
      const float r1 = rng.draw();
      if (r1 < hp * (1.0f + 1.5f * fabsf(mu))) {
        p.itype = 2;
        totevelo = totevelo + p.e * (1.0 - (double)elabfact);
        p.e = p.e * (double)elabfact;
        p.e0 = p.e0 * (double)elabfact;
        wl = __fdividef(wl, elabfact);
        ix = l;
      } else {
        const float a = rng.draw(), b = rng.draw();
        const float m = a > b ? a : b;
        mu = out ? -m : m;
        mu = aberrate(mu, vx * cinvf);
        p.x = edge;
        vx = (float)(out ? R.vxb : R.vxa);
      }
    }
  } else {  // Doppler shift
    if (dvdr > 0.f) {
      if (ig < A.ng) {
        ig = ig + 1;
        wl = (float)((A.wl[ig - 1] + 1e-6 * (A.wl[ig] - A.wl[ig - 1])) * (double)elabfactold);
      } else {
        const float r1 = rng.draw();
        wl = 1.0f / (r1 * (float)A.wlinv[A.ng] + (1.0f - r1) * (float)A.wlinv[A.ng - 1]) * elabfact;
      }
    } else if (dvdr < 0.f) {
      if (ig > 1) {
        wl = (float)((A.wl[ig - 1] + 1e-6 * (A.wl[ig - 2] - A.wl[ig - 1])) * (double)elabfactold);
        ig = ig - 1;
      } else {
        const float r1 = rng.draw();
        wl = 1.0f / (r1 * (float)A.wlinv[0] + (1.0f - r1) * (float)A.wlinv[1]) * elabfact;
      }
    }
    if (((sigc + capf(A, ig, gc + 1)) * R.dist >= (float)A.tauddmc) && !A.puretran) {
      p.itype = 2;
      totevelo = totevelo + p.e * (double)(vx * mu * cinvf);
      p.e = p.e * (double)elabfact;
      p.e0 = p.e0 * (double)elabfact;
      wl = wl / elabfact;
    }
  }
}

// one DDMC event (diffusion11.f90) in mixed precision
__device__ inline void diffusion11_mix(const TrnArgs& A, const MView& v, PtclM& p, PhiloxStream32& rng,
                                       double& eraddens,
                                       double& totevelo, int& ierr) {
  const int ng = A.ng;
  int& ix = p.ix;
  int& ig = p.ig;
  float& mu = p.mu;
  float& wl = p.wl;
  float& vx = p.vx;
  const int ic = ix;
  const int gc = v.co + ic - 1;  // 0-based index of the cell over all models
  const MixCell& R = A.mcell[gc];  // this shell's record (one line), read where needed
  ierr = 0;
  eraddens = 0.0;
  const double Xa = R.xa, Xb = R.xb;
  const size_t off = (size_t)gc * ng;
  const float divv = R.divv;
  // this group's rates in this shell (one 16-byte load); lumped groups take the
  // shell's lumped values from its record
  const float4 rt = __ldg(A.mrate + off + (ig - 1));
  if (rt.x == kRateIMC) { ierr = 100; return; }
  const int glump = rt.x == kRateLumped ? R.nlump : 0;
  float doplump, o1, o2, r_scat;
  if (glump > 0) {
    doplump = R.doplump;
    o1 = R.o1;
    o2 = R.o2;
    r_scat = glump == ng ? 0.0f : (1.0f - R.emitlump) * R.caplump;
  } else {
    doplump = rt.x;
    o1 = fabsf(rt.y);  // sign bits: the neighbour is IMC in this group
    o2 = fabsf(rt.z);
    r_scat = rt.w;
  }
  // branch rates: Doppler, left leak, right leak, effective scatter
  const float s_dop = doplump, s_left = doplump + o1, s_leak = doplump + (o1 + o2);
  const float total = s_leak + r_scat;
  const float ddmct = fabsf(__fdividef(__logf(rng.draw()), total) * cinvf);
  eraddens = p.e * (double)ddmct;
  const float u = rng.draw() * total;  // < total: r < 1 rounds below
  const int16_t* glumps = A.T.glumps + off;
  int iiig;
  if (u < s_dop) {
    if (glump == 0) {
      iiig = ig;
    } else {
      const int q = cdf_search32(A.T, 0, gc, A.T.cdf32_dop + off, glump, rng.draw());
      iiig = divv >= 0.f ? glumps[q] : glumps[glump - 1 - q];
    }
    if (divv >= 0.f) {
      ig = iiig + 1;
      wl = (float)A.wl[ig - 1];
      ig = ig < ng ? ig : ng;
    } else {
      ig = iiig - 1;
      wl = (float)A.wl[ig];
      ig = ig > 1 ? ig : 1;
    }
    if (__ldg(&A.mrate[off + ig - 1].x) == kRateIMC) {
      p.itype = 1;
      mu = 1.0f - 2.0f * rng.draw();
      const double rr = (double)rng.draw();
      double x = pow(rr * cube(Xb) + (1.0 - rr) * cube(Xa), third_r4);
      x = x < Xb ? x : Xb;
      x = x > Xa ? x : Xa;
      p.x = x;
      vx = (float)((R.vxa * (Xb - x) + R.vxb * (x - Xa)) / (Xb - Xa));
      mu = aberrate(mu, vx * cinvf);
      const float f = 1.0f - vx * mu * cinvf;
      wl = wl * f;
      const double help = 1.0 / (double)f;
      totevelo = totevelo + p.e * (1.0 - help);
      p.e = p.e * help;
      p.e0 = p.e0 * help;
    }
  } else if (u < s_leak) {
    const bool right = u >= s_left;
    p.idist = right ? -4 : -3;
    if (!right && ix == 1) return;
    if (right && ix == v.nx) {
      p.stat = 1;
      const float a = rng.draw(), b = rng.draw();
      mu = a > b ? a : b;
      if (glump != 0) ig = glumps[cdf_search32(A.T, 2, gc, A.T.cdf32_right + off, glump, rng.draw())];
      const float r = rng.draw();
      wl = 1.0f / (r * (float)A.wlinv[ig] + (1.0f - r) * (float)A.wlinv[ig - 1]);
      p.x = Xb;  // ix == nx
      vx = (float)R.vxb;
      mu = aberrate(mu, vx * cinvf);
      mu = mu < 1.0f ? mu : 1.0f;
      const double help = 1.0 / (double)(1.0f - mu * vx * cinvf);
      totevelo = totevelo + p.e * (1.0 - help);
      wl = wl / (float)help;
      p.e = p.e * help;
      p.e0 = p.e0 * help;
      return;
    }
    const int l = right ? ix + 1 : ix - 1;
    iiig = glump == 0 ? ig
                      : glumps[cdf_search32(A.T, right ? 2 : 1, gc,
                                            (right ? A.T.cdf32_right : A.T.cdf32_left) + off, glump, rng.draw())];
    // IMC in the neighbour for the group that leaks: the sign bit of this
    // group's leak rate, or the neighbour's rate sentinel for a resolved group
    const bool to_imc = glump == 0 ? signbit(right ? rt.z : rt.y)
                                   : __ldg(&A.mrate[(size_t)(v.co + l - 1) * ng + iiig - 1].x) == kRateIMC;
    if (to_imc) {
      p.itype = 1;
      const float r = rng.draw();
      wl = 1.0f / (r * (float)A.wlinv[iiig] + (1.0f - r) * (float)A.wlinv[iiig - 1]);
      p.x = right ? Xb : Xa;
      vx = (float)(right ? R.vxb : R.vxa);
      const float a = rng.draw(), b = rng.draw();
      const float m = a > b ? a : b;
      mu = right ? m : -m;
      mu = aberrate(mu, vx * cinvf);
      const float f = 1.0f - vx * mu * cinvf;
      const double help = 1.0 / (double)f;
      totevelo = totevelo + p.e * (1.0 - help);
      p.e = p.e * help;
      p.e0 = p.e0 * help;
      wl = wl * f;
    }
    ix = l;
    ig = iiig;
  } else {
    p.idist = -2;
    if (glump == ng) { ierr = 102; return; }
    if (glump == 0) {
      iiig = emitgroup_mix(A, gc, rng.draw());
    } else {
      const int q = cdf_search32(A.T, 3, gc, A.T.cdf32_scat + off, ng - glump, rng.draw());
      iiig = glumps[ng - 1 - q];
    }
    ig = iiig;
    if (__ldg(&A.mrate[off + ig - 1].x) == kRateIMC) {
      p.itype = 1;
      const float r = rng.draw();
      wl = 1.0f / ((1.0f - r) * (float)A.wlinv[ig - 1] + r * (float)A.wlinv[ig]);
      mu = 1.0f - 2.0f * rng.draw();
      const double rr = (double)rng.draw();
      double x = pow(rr * cube(Xb) + (1.0 - rr) * cube(Xa), third_r4);
      x = x < Xb ? x : Xb;
      x = x > Xa ? x : Xa;
      p.x = x;
      vx = (float)((R.vxa * (Xb - x) + R.vxb * (x - Xa)) / (Xb - Xa));
      mu = aberrate(mu, vx * cinvf);
      const float f = 1.0f - vx * mu * cinvf;
      const double help = 1.0 / (double)f;
      totevelo = totevelo + p.e * (1.0 - help);
      p.e = p.e * help;
      p.e0 = p.e0 * help;
      wl = wl * f;
    }
  }
  if (p.x < R.x0) { p.stat = 2; return; }
  const float dv = ix == ic ? divv : (float)A.divv[v.co + ix - 1];  // the shell after a leak
  const double decay = (double)__expf(-dv * ddmct * (1.0f / 3.0f));
  totevelo = totevelo + p.e * (1.0 - decay);
  p.e = p.e * decay;
  p.e0 = p.e0 * decay;
}

// DDMC branch rates of every (cell, group), as diffusion11_mix formed them per
// event (diffusion11.f90:154-231): for an unlumped group {doplump,
// opacleak(1), opacleak(2), (1 - emitlump) caplump}, the Planck factors in FP64
// rounded once, the leakage coefficients in FP32; the sign bit of opacleak(1)
// / opacleak(2) set when the left / right neighbour is IMC in this group.  A
// lumped group (cap dist >= taulump in a shell with lumped groups) gets
// kRateLumped, a group with (sig + cap) dist < tauddmc kRateIMC (the sanity
// check of :164-167).  One thread per entry; nc cells over all models.
__global__ void mix_rate_kernel(const TrnArgs A, int nc, const int4* __restrict__ cellmap, float4* __restrict__ out) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int ng = A.ng;
  if (k >= (size_t)nc * ng) return;
  const int c = (int)(k / ng), ig = (int)(k - (size_t)c * ng) + 1;
  int i = c + 1, nx = nc;
  if (cellmap) {
    const int4 cm = cellmap[c];
    i = cm.x;
    nx = cm.y;
  }
  const MixCell& R = A.mcell[c];
  const float tau_l = (float)A.taulump, tau_d = (float)A.tauddmc;
  const float capc = A.cap[k], dist = R.dist, sigc = R.sig;
  float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
  if ((sigc + capc) * dist < tau_d) {
    r.x = kRateIMC;
  } else if (capc * dist >= tau_l && R.nlump > 0) {
    r.x = kRateLumped;
  } else {
    const double tinv = R.tinv;
    const float emitlump = (float)(specint0(tinv, A.wlinv, ig) * R.capgreyinv * (double)capc);
    const double spec_ig = A.T.specarr[k];
    const double divvd = A.divv[c];
    float doplump;
    if (ig != ng && R.divv >= 0.f) doplump = (float)(dopspeccalc(tinv, A.wlinv, ig) * divvd / (spec_ig * 3.0 * pc_c));
    else if (ig != 1 && R.divv < 0.f) doplump = (float)(-dopspeccalc(tinv, A.wlinv, ig - 1) * divvd / (spec_ig * 3.0 * pc_c));
    else doplump = 0.f;
    float o1 = 0.f, o2;
    bool left_imc = false, right_imc = false;
    if (i > 1) {
      const float capl = A.cap[k - ng];
      if ((capl + R.sigl) * R.dxl < tau_d) {
        const float ppl = 4.0f / (3.0f * (capc + sigc) * dist + 6.0f * dextf);
        o1 = 1.5f * ppl * R.fa;
        left_imc = true;
      } else {
        o1 = 2.0f * R.fa / ((sigc + capc) * dist + (R.sigl + capl) * R.dxl);
      }
    }
    bool lhelp = true;
    float capl = 0.f;
    if (i != nx) {
      capl = A.cap[k + ng];
      lhelp = (capl + R.sigr) * R.dxr < tau_d;
      right_imc = lhelp;
    }
    if (lhelp) {
      const float ppr = 4.0f / (3.0f * (capc + sigc) * dist + 6.0f * dextf);
      o2 = 1.5f * ppr * R.fb;
    } else {
      o2 = 2.0f * R.fb / ((sigc + capc) * dist + (R.sigr + capl) * R.dxr);
    }
    r.x = doplump;
    r.y = left_imc ? -o1 : o1;
    r.z = right_imc ? -o2 : o2;
    r.w = (1.0f - emitlump) * capc;
  }
  out[k] = r;
}

// Emission CDF of every cell over its groups: running sums of specarr * cap in
// group order (the order of emitprob's bins and of emitgroup's walk inside a
// bin, emitgroup.f:3-54) divided by capgrey, in FP32, and the guide table of
// the running sums (entry k = number of sums <= k / guide_m).  One block per cell.
__global__ void mix_emit_kernel(const TrnArgs A, float* __restrict__ cdf, int16_t* __restrict__ guide) {
  const int c = blockIdx.x, ng = A.ng, gm = A.T.guide_m;
  float* a = cdf + (size_t)c * ng;
  if (threadIdx.x == 0) {
    const double inv = 1.0 / A.capgrey[c];
    const double* sp = A.T.specarr + (size_t)c * ng;
    const float* cp = A.cap + (size_t)c * ng;
    double s = 0.0;
    for (int g = 0; g < ng; ++g) {
      s = s + sp[g] * (double)cp[g];
      a[g] = (float)(s * inv);
    }
  }
  __syncthreads();
  int16_t* gd = guide + (size_t)c * (gm + 1);
  for (int k = threadIdx.x; k <= gm; k += blockDim.x) {
    const float v = (float)k / (float)gm;  // exact: gm is a power of two
    int lo = 0, hi = ng;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (a[mid] <= v) lo = mid + 1;
      else hi = mid;
    }
    gd[k] = (int16_t)lo;
  }
}

template <int MINB>
__global__ void __launch_bounds__(MIX_BLOCK, MINB) particle_advance_mixed_kernel(const TrnArgs A) {
  __shared__ unsigned long long s_cnt[20];
  __shared__ double s_sum[3];
  // grd_tally of the whole grid in shared memory when it fits (A.smem_cells
  // cells): a DDMC walk changes shell on almost every event, and flushing
  // each visit to the few hundred global tally words made the warps wait on
  // contended L2 atomics
  extern __shared__ double s_tally[];
  if (threadIdx.x < 20) s_cnt[threadIdx.x] = 0ull;
  if (threadIdx.x < 3) s_sum[threadIdx.x] = 0.0;
  for (int k = threadIdx.x; k < A.smem_cells; k += blockDim.x) s_tally[k] = 0.0;
  __syncthreads();
  double* const tally = A.smem_cells ? s_tally : A.tally;
  const int lane = threadIdx.x & 31;
  // counters are kept per particle in 32 bits (DDMC steps, method swaps; the
  // IMC steps are istep - nd_p) and added to the block's shared counters when
  // the particle ends, so few registers carry them through the loop
  double evelo = 0.0;
  unsigned nd_p = 0, nsw_p = 0;
  long long ip = -1;
  bool have = false, queue_done = false;
  PtclM p;
  PhiloxStream32 rng;
  // replays of a captured graph draw from counter word 3 = 2 | replay << 2
  const uint32_t sw = 2u | (A.epoch ? (uint32_t)(*A.epoch << 2) : 0u);
  // the current particle's model (plain integers: a struct updated member by
  // member in the refill branch lost its shell count on sm_100a builds)
  int vnx = A.nx, vco = 0, vxo = 0;
  int istep = 0;
  int t_ic = 0, j_ic = 0, j_ig = 0;
  double t_acc = 0.0, t_c = 0.0, j_acc = 0.0, j_c = 0.0;
  while (true) {
    __syncwarp();
    const bool need = !have && !queue_done;
    const unsigned needm = __ballot_sync(0xffffffffu, need);
    if (needm) {
      const int leader = __ffs(needm) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(&A.acc->next, (unsigned long long)__popc(needm));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const long long cand = (long long)base + __popc(needm & ((1u << lane) - 1u));
        if (cand >= A.npart) {
          queue_done = true;
        } else if (!A.isvacant[cand]) {
          ip = cand;
          const double2* q = reinterpret_cast<const double2*>(A.prt + ip);
          const double2 b = q[1], c = q[2], d = q[3];
          double x = A.prt[ip].x, mu = b.y, e = c.y, e0 = d.x, wl = d.y;
          atomicAdd(&s_cnt[0], 1ull);
          // the slot's model (models own consecutive slot ranges)
          int m = 0;
          long long poff = 0;
          if (A.nmodel > 1) {
            int lo = 0, hi = A.nmodel - 1;
            while (lo < hi) {
              const int mid = (lo + hi + 1) >> 1;
              if (__ldg(&A.models[mid].poff) <= ip) lo = mid;
              else hi = mid - 1;
            }
            m = lo;
            poff = __ldg(&A.models[m].poff);
            vnx = __ldg(&A.models[m].nx);
            vco = __ldg(&A.models[m].co);
            vxo = __ldg(&A.models[m].xo);
          }
          const double* X = A.xarr + vxo;
          const double* VX = A.vxarr + vxo;
          int ix = binsrch(x, X, vnx + 1, false);
          int ig = binsrch(wl, A.wl, A.ng + 1, false);
          if (ix < 1 || ig < 1) {
            if (A.errorfatal) atomicMin(&A.acc->ierr_key, ((unsigned long long)(ip + 1) << 32) | 1002u);
            A.isvacant[ip] = 1;
          } else {
            const double tau = (A.sig[vco + ix - 1] + CAPd(A, ig, vco + ix)) * (X[ix] - X[ix - 1]);
            p.itype = (A.puretran || tau < A.tauddmc) ? 1 : 2;
            const double vx = (VX[ix - 1] * (X[ix] - x) + VX[ix] * (x - X[ix - 1])) / (X[ix] - X[ix - 1]);
            if (p.itype == 1) {
              const double labfact = 1.0 - vx * mu / pc_c;
              wl = wl * labfact;
              e = e / labfact;
              e0 = e0 / labfact;
            }
            p.x = x; p.e = e; p.e0 = e0; p.mu = (float)mu; p.wl = (float)wl; p.vx = (float)vx;
            p.ix = ix; p.ig = ig; p.stat = 0; p.idist = 0;
            istep = 0;
            nd_p = 0;
            nsw_p = 0;
            rng.init(A.seed + (unsigned long long)m * kModelSeedStride, (uint64_t)(ip - poff), sw);
            have = true;
          }
        }
      }
    }
    if (__all_sync(0xffffffffu, !have && queue_done)) break;
    if (!have) continue;
    istep++;
    rng.begin_event((uint32_t)istep);
    const MView v{vnx, vco, vxo};
    const int icold = v.co + p.ix, igold = p.ig;  // cell over all models, 1-based
    double eraddens;
    int ierr;
    if (p.itype == 1 || A.puretran) {
      transport11_mix(A, v, p, rng, eraddens, evelo, ierr);
      if (p.itype != 1) {
        nsw_p++;
        if (A.dogrdtally) atomicAdd(&A.methodswap[icold - 1], 1);
      }
    } else {
      nd_p++;
      diffusion11_mix(A, v, p, rng, eraddens, evelo, ierr);
      if (p.itype == 1) {
        nsw_p++;
        if (A.dogrdtally) atomicAdd(&A.methodswap[icold - 1], 1);
      }
    }
    {
      // ndist histogram: one shared-memory add per distinct bin in the warp
      const int di = 9 + (p.idist > -3 ? p.idist : -3) + 3;
      const unsigned grp = __match_any_sync(__activemask(), di);
      if (lane == __ffs(grp) - 1) atomicAdd(&s_cnt[di], (unsigned long long)__popc(grp));
    }
    if (icold != t_ic) {
      if (t_ic > 0) atomicAdd(&tally[t_ic - 1], t_acc - t_c);
      t_ic = icold;
      t_acc = 0.0;
      t_c = 0.0;
    }
    kahan_add(t_acc, t_c, eraddens);
    if (icold != j_ic || igold != j_ig) {
      if (j_ic > 0) atomicAdd(&A.jrad[(size_t)(j_ic - 1) * A.ng + (j_ig - 1)], pc_c * (j_acc - j_c));
      j_ic = icold;
      j_ig = igold;
      j_acc = 0.0;
      j_c = 0.0;
    }
    kahan_add(j_acc, j_c, eraddens);
    if (p.itype == 1 && p.stat == 0) {
      if (p.x > A.xarr[v.xo + p.ix] || p.x < A.xarr[v.xo + p.ix - 1] || p.x != p.x) {
        if (ierr == 0) ierr = -99;
      }
    }
    if (ierr == -99) atomicAdd(&s_cnt[6], 1ull);
    if (ierr == 0 && A.max_steps > 0 && istep >= A.max_steps && p.stat == 0) ierr = 1001;
    if (ierr > 0) {
      if (A.errorfatal) atomicMin(&A.acc->ierr_key, ((unsigned long long)(ip + 1) << 32) | (unsigned)ierr);
      p.stat = 2;
    }
    if (p.stat != 0) {
      atomicMax(&s_cnt[5], (unsigned long long)istep);
      atomicAdd(&s_cnt[2], (unsigned long long)(istep - nd_p));
      atomicAdd(&s_cnt[3], (unsigned long long)nd_p);
      if (nsw_p) atomicAdd(&s_cnt[4], (unsigned long long)nsw_p);
      if (p.stat == 2) {
        A.isvacant[ip] = 1;
      } else {
        atomicAdd(&s_cnt[1], 1ull);
        atomicAdd(&s_sum[1], p.e);   // tot_eout
        atomicAdd(&s_sum[2], -p.e);  // tot_sflux
        // y, z and om are never changed in the slot
        slg_packet* q = A.prt + ip;
        q->x = DBL_MAX;
        q->mu = (double)p.mu;
        q->e = p.e;
        reinterpret_cast<double2*>(q)[3] = make_double2(p.e0, (double)p.wl);
      }
      have = false;
    }
  }
  if (t_ic > 0) atomicAdd(&tally[t_ic - 1], t_acc - t_c);
  if (j_ic > 0) atomicAdd(&A.jrad[(size_t)(j_ic - 1) * A.ng + (j_ig - 1)], pc_c * (j_acc - j_c));
  atomicAdd(&s_sum[0], evelo);
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicAdd(&A.acc->evelo, s_sum[0]);
    atomicAdd(&A.acc->eout, s_sum[1]);
    atomicAdd(&A.acc->sflux, s_sum[2]);
    atomicAdd(&A.acc->npckt, s_cnt[0]);
    atomicAdd(&A.acc->nflux, s_cnt[1]);
    atomicAdd(&A.acc->nimc, s_cnt[2]);
    atomicAdd(&A.acc->nddmc, s_cnt[3]);
    atomicAdd(&A.acc->nswap, s_cnt[4]);
    atomicMax(&A.acc->nmax, s_cnt[5]);
    atomicAdd(&A.acc->nwarn, s_cnt[6]);
  }
  if (threadIdx.x < 11 && s_cnt[9 + threadIdx.x]) atomicAdd(&A.acc->ndist[threadIdx.x], s_cnt[9 + threadIdx.x]);
  for (int k = threadIdx.x; k < A.smem_cells; k += blockDim.x)
    if (s_tally[k] != 0.0) atomicAdd(&A.tally[k], s_tally[k]);
}

template <int MINB>
int launch_mixed_one(int num_sms, long long npart, cudaStream_t st, const TrnArgs& A) {
  // resident blocks per SM, queried again only when the shared tally size changes
  static int occ = -1;
  static size_t occ_shm = 0;
  const size_t shm = sizeof(double) * (size_t)A.smem_cells;
  if (occ < 0 || shm != occ_shm) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, particle_advance_mixed_kernel<MINB>, MIX_BLOCK, shm);
    occ_shm = shm;
  }
  long long nblk = (long long)num_sms * (occ > 0 ? occ : 1);
  const long long need = (npart + MIX_BLOCK - 1) / MIX_BLOCK;
  if (need < nblk) nblk = need > 0 ? need : 1;
  particle_advance_mixed_kernel<MINB><<<(unsigned)nblk, MIX_BLOCK, shm, st>>>(A);
  return cudaPeekAtLastError() == cudaSuccess ? SLG_OK : SLG_ERR_CUDA;
}

}  // namespace

// The per-(cell, group) rate table and the emission CDF of a mixed-precision
// launch (A.mcell, A.T.specarr and the opacities must be in place).
int launch_mix_rate_tables(cudaStream_t st, int nc, const int4* cellmap, const TrnArgs& A, float4* mrate,
                           float* emit32, int16_t* eguide) {
  const size_t n = (size_t)nc * A.ng;
  mix_rate_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(A, nc, cellmap, mrate);
  mix_emit_kernel<<<nc, 128, 0, st>>>(A, emit32, eguide);
  return cudaPeekAtLastError() == cudaSuccess ? SLG_OK : SLG_ERR_CUDA;
}

// Variants: resident 128-thread blocks per SM requested from the compiler
// (register budget 128 / 102 / 85 / 73 per thread).
int launch_transport_mixed(int variant, int num_sms, long long npart, cudaStream_t st, const TrnArgs& A) {
  switch (variant) {
    case 1: return launch_mixed_one<5>(num_sms, npart, st, A);
    case 2: return launch_mixed_one<6>(num_sms, npart, st, A);
    case 3: return launch_mixed_one<7>(num_sms, npart, st, A);
    default: return launch_mixed_one<4>(num_sms, npart, st, A);
  }
}

}  // namespace slg
