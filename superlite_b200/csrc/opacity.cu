// opacity.cu -- physical LTE opacity (bound-bound expansion opacity binned into
// groups, Verner bound-free, Sutherland free-free), analytic opacity and the
// Planck / Rosseland means, for sm_100a.
//
// Reference: GAS/physical_opacity.f:3-357, bfxsmod.f:65-153,
// GAS/analytic_opacity.f90:3-77, GAS/opacity_planckmean.f:17-24,
// GAS/opacity_rossmean.f:17-21.
//
// Design (one B200):
//  * bin_lines: lines (sorted by wl0) are binned to sub-groups by a
//    warp-cooperative kernel: the sub-group edges are staged into shared memory
//    with one TMA bulk copy (cp.async.bulk + mbarrier), each thread binary-
//    searches its lines there, and a shared-memory histogram of lines per
//    sub-group is flushed to global counts; a scan turns counts into ranges.
//  * opacity_fwd: one warp per (group, 32 shells).  Every lane walks the
//    lines of its group in file order (warp-uniform broadcast reads) and
//    accumulates bb, then bf (ions in the reference's iz,ii order), then ff
//    (elements in order) into one register, i.e. exactly the reference's
//    per-(cell,sub-group) summation order.  Sub-groups are collapsed in
//    registers, then cap and emissivity are written through a shared-memory
//    tile so each shell's 8 groups leave as one 32-byte sector.
//  * FP64 throughout, no FMA contraction (-fmad=false), so sums round like the
//    single-threaded Fortran; only exp/log10/pow may differ in the last ulp.
#include <cuda_runtime.h>
#include <cfloat>
#include "slg_device.cuh"
#include "slg_internal.h"

namespace slg {

namespace {

constexpr int OPAC_GT = 8;   // groups per block (one warp each)
constexpr int OPAC_CT = 32;  // shells per block (one per lane)
// forward: FS shells per lane (a block covers FS * OPAC_CT shells), 2 or 4
// (opacity_fwd_kernel<FS>; launch_fwd picks it)

// ------------------------------------------------------------ TMA bulk helpers
__device__ inline uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ inline void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ inline void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ inline void tma_bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Bounded wait on phase 0 of the barrier.  Returns false on time-out.
__device__ inline bool mbar_wait(uint64_t* bar, uint32_t parity, long max_polls) {
  for (long it = 0; it < max_polls; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    if (it > 64) __nanosleep(64);
  }
  return false;
}

// ------------------------------------------------------------ line binning
// counts[igs] (igs = 0..ngsub+1) = number of lines whose sub-group pointer is
// igs (physical_opacity.f:117-125): igs = #{k : wlsub(k) <= wl0}.
__global__ void __launch_bounds__(256) bin_lines_kernel(const slg_bbxs* __restrict__ bb, int64_t nline,
                                                        const double* __restrict__ wlsub_pad,
                                                        int nedge, int nedge_pad,
                                                        unsigned int* __restrict__ counts,
                                                        int* __restrict__ flags) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  double* edges = reinterpret_cast<double*>(smem + 16);
  unsigned int* hist = reinterpret_cast<unsigned int*>(smem + 16 + sizeof(double) * nedge_pad);
  const int nbins = nedge + 1;  // 0..ngsub+1
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_expect_tx(bar, (uint32_t)(sizeof(double) * nedge_pad));
    tma_bulk_g2s(edges, wlsub_pad, (uint32_t)(sizeof(double) * nedge_pad), bar);
  }
  for (int k = threadIdx.x; k < nbins; k += blockDim.x) hist[k] = 0u;
  __syncthreads();
  if (!mbar_wait(bar, 0, 1L << 24)) {
    if (threadIdx.x == 0) atomicOr(flags + 1, 2);
    // keep waiting (bounded) for the copy in flight before leaving
    mbar_wait(bar, 0, 1L << 24);
    return;
  }
  const int64_t per_block = (int64_t)blockDim.x * 8;
  const int64_t l0 = (int64_t)blockIdx.x * per_block;
  for (int it = 0; it < 8; ++it) {
    const int64_t l = l0 + (int64_t)it * blockDim.x + threadIdx.x;
    if (l >= nline) break;
    const float w = bb[l].wl0;
    if (l + 1 < nline && !(w <= bb[l + 1].wl0)) atomicOr(flags + 1, 1);
    const double wl0 = (double)w * pc_ang;
    // upper bound: number of edges <= wl0
    int lo = 0, hi = nedge;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (edges[mid] <= wl0) lo = mid + 1;
      else hi = mid;
    }
    atomicAdd(&hist[lo], 1u);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < nbins; k += blockDim.x)
    if (hist[k]) atomicAdd(&counts[k], hist[k]);
}

// exclusive scan of counts (n <= a few 1e4) in one block
__global__ void __launch_bounds__(1024) scan_counts_kernel(const unsigned int* __restrict__ counts, int n,
                                                           int* __restrict__ start) {
  __shared__ int part[1024];
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int b = threadIdx.x * per;
  int s = 0;
  for (int k = b; k < b + per && k < n; ++k) s += (int)counts[k];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int t = 0; t < (int)blockDim.x; ++t) {
      const int v = part[t];
      part[t] = acc;
      acc += v;
    }
  }
  __syncthreads();
  int acc = part[threadIdx.x];
  for (int k = b; k < b + per && k < n; ++k) {
    start[k] = acc;
    acc += (int)counts[k];
  }
  if (threadIdx.x == blockDim.x - 1) start[n] = acc;
}

// ------------------------------------------------------------ per-cell preparation
// hckt (physical_opacity.f:81), gas_sig (:84-89), hlparr (:203), grndlev (:95-101,
// :165-171) and the per-(cell,element) free-free Gaunt row indices (:226-231).
__global__ void opac_cell_prep_kernel(int nc, int nelem, int nst, const int32_t* __restrict__ ion_ni,
                                      const double* __restrict__ temp, const double* __restrict__ natom,
                                      const double* __restrict__ nelec, const double* __restrict__ vol,
                                      const double* __restrict__ mass, const double* __restrict__ oc,
                                      const double* __restrict__ ginv, int nothmson,
                                      double* __restrict__ hckt, double* __restrict__ gas_sig,
                                      double* __restrict__ hlparr, double* __restrict__ grndlev,
                                      int* __restrict__ ffigg, double* __restrict__ ffdgg) {
  // one thread per (shell i, element iz = blockIdx.y + 1)
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nc) return;
  const double h = pc_hc / (pc_kb * temp[i]);
  if (blockIdx.y == 0) {
    hckt[i] = h;
    double s = 0.0;
    if (!nothmson) {
      s = cthomson * nelec[i] * natom[i] / vol[i];
      if (mass[i] <= 0.0) s = 0.0;
    }
    gas_sig[i] = s;
    hlparr[i] = sq(natom[i] / vol[i]) * nelec[i];
  }
  {
    const int iz = blockIdx.y + 1;
    const int lim = min(iz, ion_ni[iz - 1] - 1);
    for (int ii = 1; ii <= nst; ++ii) {
      const size_t k = (size_t)(iz - 1) * nst + (ii - 1);
      double v = 0.0;
      if (ii <= lim && mass[i] > 0.0) v = oc[k * nc + i] * ginv[k * nc + i];
      grndlev[k * nc + i] = v;
    }
    const double gg = (double)(iz * iz) * pc_rydberg * h;
    const double rgg = 5.0 * (log10(gg) + 4.0) + 1.0;
    // max(floor(rgg), 1) and min(., ff_ngg - 1) as :228-230; a NaN (from a NaN
    // temperature) takes the lower bound, so the table reads stay in bounds
    int igg = !(rgg >= 1.0) ? 1 : (rgg >= (double)(FF_NGG - 1) ? FF_NGG - 1 : (int)floor(rgg));
    ffigg[(size_t)(iz - 1) * nc + i] = rgg > (double)FF_NGG ? -igg : igg;  // sign: gff >= 1 clamp (:238)
    ffdgg[(size_t)(iz - 1) * nc + i] = rgg - igg;
  }
}

// Free-free, summed over elements once per shell.  For fixed table columns
// (igg, dgg) of each element, the reference's bilinear gff (physical_opacity.f:
// 234-237) is linear in the row weights (1 - du, du):
//   g_z = (1 - du) Gz[iu - 1] + du Gz[iu],  Gz[j] = (1 - dgg) G[j, igg - 1] + dgg G[j, igg],
// so sum_z z^2 fr_z g_z = (1 - du) S[iu - 1] + du S[iu] with
// S[j] = sum_z z^2 fr_z Gz[j] over the elements without the gff >= 1 clamp
// (:238, nonlinear); those are flagged in ffclamp (bit iz - 1) and added per
// group.  Elements with fr = 0 add +0 in the reference (:240-241) and are left
// out.  The sum is re-associated (one product by help per group instead of one
// per element): a rounding-level difference.  For the adjoint: D[j] = sum_z
// z^2 fr_z (G[j, igg] - G[j, igg - 1]) over the same elements (d gff / d dgg
// is linear in the row weights too), and ffclamp_all flags every clamped
// element whatever its fr (d cap / d fr needs them all).
// One thread per (shell, table row j).
__global__ void ff_sum_kernel(int nc, int nelem, const double* __restrict__ natomfr, const int* __restrict__ ffigg,
                              const double* __restrict__ ffdgg, const double* __restrict__ G,
                              double* __restrict__ ffsum, double* __restrict__ ffdsum, unsigned* __restrict__ ffclamp,
                              unsigned* __restrict__ ffclamp_all) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nc * FF_NU) return;
  const int i = (int)(t / FF_NU), j = (int)(t % FF_NU);
  const double* nfr = natomfr + (size_t)(nelem + 1) * i;
  double S = 0.0, D = 0.0;
  unsigned clamp = 0, clamp_all = 0;
  for (int iz = 1; iz <= nelem; ++iz) {
    const double fr = nfr[iz];
    const int igg = ffigg[(size_t)(iz - 1) * nc + i];
    if (igg < 0) {
      clamp_all |= 1u << (iz - 1);
      if (fr != 0.0) clamp |= 1u << (iz - 1);
      continue;
    }
    if (fr == 0.0) continue;
    const double dgg = ffdgg[(size_t)(iz - 1) * nc + i];
    const double g0 = G[j + FF_NU * (igg - 1)], g1 = G[j + FF_NU * igg];
    const double gz = (1.0 - dgg) * g0 + dgg * g1;
    const double w = (double)(iz * iz) * fr;
    S = S + w * gz;
    D = D + w * (g1 - g0);
  }
  ffsum[(size_t)i * FF_NU + j] = S;
  ffdsum[(size_t)i * FF_NU + j] = D;
  if (j == 0) {
    ffclamp[i] = clamp;
    ffclamp_all[i] = clamp_all;
  }
}

// Which ion slots (iz,ii) carry any population: 1 if any cell has oc != 0.
__global__ void ion_active_kernel(int nc, const double* __restrict__ oc, int* __restrict__ active) {
  const int k = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x)
    if (oc[(size_t)k * nc + i] != 0.0) { active[k] = 1; return; }
}

// Active slots in the reference's loop order (iz ascending, ii = 1..min(iz,ni-1)),
// physical_opacity.f:180-181: that order is increasing slot = (iz-1) nst + (ii-1),
// so one warp compacts the valid, populated slots 32 at a time with a ballot.
__global__ void ion_compact_kernel(int nelem, int nst, const int32_t* __restrict__ ion_ni,
                                   const int* __restrict__ active, int16_t* __restrict__ act_slot,
                                   int* __restrict__ nact) {
  const int lane = threadIdx.x & 31;
  const int nslot = nelem * nst;
  int n = 0;
  for (int k0 = 0; k0 < nslot; k0 += 32) {
    const int k = k0 + lane;
    bool ok = false;
    if (k < nslot) {
      const int iz = k / nst + 1, ii = k % nst + 1;
      ok = ii <= min(iz, ion_ni[iz - 1] - 1) && active[k] != 0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if (ok) act_slot[n + __popc(m & ((1u << lane) - 1u))] = (int16_t)k;
    n += __popc(m);
  }
  if (lane == 0) *nact = n;
}

// Sub-group edges wlsub (physical_opacity.f:65-78), padded with DBL_MAX.
__global__ void wlsub_kernel(int ng, int ngs, int nedge_pad, const double* __restrict__ wl,
                             double* __restrict__ wlsub) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;  // 0-based edge
  if (k >= nedge_pad) return;
  const int nedge = ng * ngs + 1;
  double v = DBL_MAX;
  if (k < nedge) {
    if (ngs == 1 || k == 0) {
      v = wl[ngs == 1 ? k : 0];
    } else {
      const int ig = (k - 1) / ngs + 1, i = (k - 1) % ngs + 1;
      const double help = 1.0 / ngs;
      v = (1.0 - i * help) * wl[ig - 1] + i * help * wl[ig];
    }
  }
  wlsub[k] = v;
}

// ------------------------------------------------------------ bound-free cross sections
__device__ inline float PH1(const float* t, int k, int is, int nz, int ne) {
  return t[(k - 1) + 6 * ((is - 1) + 7 * ((nz - 1) + 30 * (ne - 1)))];
}
__device__ inline float PH2(const float* t, int k, int nz, int ne) {
  return t[(k - 1) + 7 * ((nz - 1) + 30 * (ne - 1))];
}
__device__ inline float sqf(float x) { return __fmul_rn(x, x); }  // real*4 ** 2

// bfxsmod.f:65-153
__device__ double bfxs(const float* __restrict__ ph1, const float* __restrict__ ph2, int nz, int ne,
                       double e) {
  const int ll[7] = {0, 0, 1, 0, 1, 2, 0};
  const int ninn[30] = {0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 3, 3, 3, 3, 3,
                        3, 3, 3, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5};
  const int ntot[30] = {1, 1, 2, 2, 3, 3, 3, 3, 3, 3, 4, 4, 5, 5, 5,
                        5, 5, 5, 6, 6, 6, 6, 6, 6, 6, 6, 6, 6, 7, 7};
  double xs = 0.0;
  if (nz < 1 || nz > 30) return xs;
  if (ne < 1 || ne > nz) return xs;
  int nout = ntot[ne - 1];
  if (nz > 18) {
    if (nz == ne) nout = 7;
    if (nz == ne + 1 && (nz == 20 || nz == 21 || nz == 22 || nz == 25 || nz == 26)) nout = 7;
  }
  if (e < (double)PH1(ph1, 1, nout, nz, ne)) return xs;
  const int nint_ = ninn[ne - 1];
  double einn;
  if (nz == 15 || nz == 17 || nz == 19 || (nz > 20 && nz != 26)) einn = 0.0;
  else einn = ne < 3 ? (double)1.0e30f : (double)PH1(ph1, 1, nint_, nz, ne);
  for (int is = 1; is <= nout; ++is) {
    if (e < (double)PH1(ph1, 1, is, nz, ne)) continue;
    if (is < nout && is > nint_ && e < einn) continue;
    if (is <= nint_ || e >= einn) {
      const double p1 = -(double)PH1(ph1, 5, is, nz, ne);
      const double y = e / (double)PH1(ph1, 2, is, nz, ne);
      const double q = -0.5 * p1 - (double)ll[is - 1] - 5.5;
      const double a = (double)PH1(ph1, 3, is, nz, ne) * (sq(y - 1.0) + (double)sqf(PH1(ph1, 6, is, nz, ne)));
      const double b = sqrt(y / (double)PH1(ph1, 4, is, nz, ne)) + 1.0;
      xs = xs + a * pow(y, q) * pow(b, p1);
    } else {
      const double p1 = -(double)PH2(ph2, 4, nz, ne);
      const double q = -0.5 * p1 - 5.5;
      const double x = e / (double)PH2(ph2, 1, nz, ne) - (double)PH2(ph2, 6, nz, ne);
      const double z = sqrt(x * x + (double)sqf(PH2(ph2, 7, nz, ne)));
      const double a = (double)PH2(ph2, 2, nz, ne) * (sq(x - 1.0) + (double)sqf(PH2(ph2, 5, nz, ne)));
      const double b = 1.0 + sqrt(z / (double)PH2(ph2, 3, nz, ne));
      xs = xs + a * pow(z, q) * pow(b, p1);
    }
  }
  return xs;
}

// xstab[(igs-1)*nact + a] = bfxs(iz, iz-ii+1, hc/(ev*wlsub(igs))), :177-183
__global__ void bf_table_kernel(int ngsub, int maxact, const int* __restrict__ pnact,
                                const int16_t* __restrict__ act_slot, int nst,
                                const double* __restrict__ wlsub, const float* __restrict__ ph1,
                                const float* __restrict__ ph2, double* __restrict__ xstab) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)ngsub * maxact) return;
  const int igs = (int)(t / maxact) + 1;
  const int a = (int)(t % maxact);
  if (a >= *pnact) return;
  const int slot = act_slot[a];
  const int iz = slot / nst + 1, ii = slot % nst + 1;
  const double wl = wlsub[igs - 1];
  const double en = pc_hc / (pc_ev * wl);
  xstab[t] = bfxs(ph1, ph2, iz, iz - ii + 1, en) * pc_mbarn;  // physical_opacity.f:185-186: xs*pc_mbarn first
}

// Per sub-group, the xstab entries with a nonzero cross section, in slot
// order (one warp per sub-group, ballot compaction): xsc = bfxs * pc_mbarn,
// bslot = the ion slot, bnnz = their count.  The reference skips xs == 0
// (physical_opacity.f:184), so summing over the compacted entries adds the
// same terms in the same order.
__global__ void bf_compact_kernel(int ngsub, int maxact, const int* __restrict__ pnact,
                                  const int16_t* __restrict__ act_slot, const double* __restrict__ xstab,
                                  double* __restrict__ xsc, int* __restrict__ bslot, int* __restrict__ bnnz) {
  const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (w >= ngsub) return;
  const int nact = *pnact;
  const size_t base = (size_t)w * maxact;
  int k = 0;
  for (int a0 = 0; a0 < nact; a0 += 32) {
    const int a = a0 + lane;
    const double x = a < nact ? xstab[base + a] : 0.0;
    const bool nz = x != 0.0;
    const unsigned m = __ballot_sync(0xffffffffu, nz);
    if (nz) {
      const int pos = k + __popc(m & ((1u << lane) - 1u));
      xsc[base + pos] = x;
      bslot[base + pos] = act_slot[a];
    }
    k += __popc(m);
  }
  if (lane == 0) bnnz[w] = k;
}

// One line's shell-independent factors, 16 bytes (one vector load per line):
// pg = phi(igs) * gxs, the first product of the reference's expression
// (physical_opacity.f:148-149), so the evaluation order of that product is
// kept; and chilw in FP64 with two indices in the low 29 bits of its
// mantissa.  chilw is single precision in the line record (as in the
// reference's bbxs type), so those bits of its FP64 value are zero: masking
// them off gives chilw exactly, without a conversion per line.  The indices:
// bits 0..10 the line's row among the population rows the lines reference
// (lrow_of_slot), bits 11..26 its population slot (iz - 1) nst + (ii - 1).
struct __align__(16) LineTerm {
  double pg;
  double chi_idx;
};
constexpr int kLineRowBits = 11;
constexpr unsigned kLineIdxMask = 0x1fffffffu;

struct LineVals {
  double pg, chi;
  unsigned idx;
};

__device__ __forceinline__ LineVals load_line(const LineTerm* p) {
  const double2 v = __ldg(reinterpret_cast<const double2*>(p));
  const unsigned lo = (unsigned)__double2loint(v.y);
  return LineVals{v.x, __hiloint2double(__double2hiint(v.y), (int)(lo & ~kLineIdxMask)), lo & kLineIdxMask};
}
__device__ __forceinline__ int line_row(unsigned idx) { return (int)(idx & ((1u << kLineRowBits) - 1)); }
__device__ __forceinline__ int line_slot(unsigned idx) { return (int)(idx >> kLineRowBits); }

// The LineTerm of each binned line of sub-groups 1..ngsub (lines outside the
// grid get zeros and are never read).
__global__ void decode_lines_kernel(const slg_bbxs* __restrict__ bb, int64_t nline, const int* __restrict__ lstart,
                                    int ngsub, const double* __restrict__ wlsub, int nst,
                                    const int16_t* __restrict__ lrow_of_slot, LineTerm* __restrict__ lt) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nline) return;
  // sub-group of line l: the largest igs with lstart[igs] <= l
  int lo = 0, hi = ngsub + 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (lstart[mid] <= l) lo = mid;
    else hi = mid - 1;
  }
  const int igs = lo;
  LineTerm t{0.0, 0.0};
  if (igs >= 1 && igs <= ngsub) {
    const slg_bbxs r = bb[l];
    const double wa = wlsub[igs - 1], wb = wlsub[igs];
    const double wl = 0.5 * (wa + wb);
    const double phi = wl * wl / ((wb - wa) * pc_c);
    const int slot = (r.iz - 1) * nst + (r.ii - 1);
    const double chi = (double)r.chilw;  // low 29 mantissa bits zero
    const unsigned idx = ((unsigned)slot << kLineRowBits) | (unsigned)lrow_of_slot[slot];
    t = LineTerm{phi * (double)r.gxs,
                 __hiloint2double(__double2hiint(chi), (int)((unsigned)__double2loint(chi) | idx))};
  }
  lt[l] = t;
}

struct OpacArgs {
  int nc, ng, ngs, ngsub, nelem, nst, maxact;
  int nobb, nobf, noff;
  const int* pnact;         // number of active bound-free ion slots (device)
  double mix;
  const double* wlsub;
  const double* grp_wl;
  const int* lstart;        // (ngsub+2)+1 offsets by igs
  const slg_bbxs* bb;
  const LineTerm* lt;       // per binned line (decode_lines_kernel)
  double chimax;            // largest chilw of the lines (infinite: check every exp argument)
  const int16_t* slot_of_lrow;  // line row -> slot
  int nlrow;                // population rows the lines reference
  int stage_rows = 0;       // forward: stage those rows of a block's shells in shared memory
  const double* grndlev;    // [slot][cell]
  const double* oc;         // [slot][cell]
  const int16_t* act_slot;  // active slots, reference order
  const double* xstab;      // [(igs-1)*maxact + a]: bfxs * pc_mbarn
  const double* xsc;        // the nonzero entries of xstab per sub-group (bf_compact_kernel)
  const int* bslot;         // their ion slots
  const int* bnnz;          // their count per sub-group
  const double* hckt;
  const double* hlparr;
  const double* mass;
  const double* natomfr;    // (0:nelem, ncell)
  const double* temp;
  const int* ffigg;         // [iz-1][cell], negative: apply gff >= 1
  const double* ffdgg;
  const double* ffsum;      // [cell][81]: sum over unclamped elements of z^2 fr gff at each table row
  const double* ffdsum;     // [cell][81]: the same of z^2 fr d gff / d dgg
  const unsigned* ffclamp;  // [cell]: elements (bit iz-1) with fr != 0 under the gff >= 1 clamp
  const unsigned* ffclamp_all;  // [cell]: every element under the clamp
  const double* gff;        // (81,41)
  double ffc1;
  float* cap32;             // (ng, ncell)
  float* emiss32;
  double* cap64;            // (ncell, ng) optional
  double* capg64 = nullptr; // (ng, ncell) optional: cap before sngl() in gas_cap's layout
  int* flags;
};

// Sum over n lines of pg * og * exp(-chi h), og the staged population of the
// line's row for this shell (s_gl: the shell's column of the block's staged
// rows, FC apart); four lines per round: their loads and exps are
// independent, and the terms are added one after another in line order, each
// by one fused multiply-add (one rounding where the reference rounds the
// product and the sum).  INRANGE: the caller has shown -chi h in [-700, 0] for
// every line.
template <bool INRANGE, int FC>
__device__ __forceinline__ double bb_sum_staged(const LineTerm* lt, int n, double h, const double* s_gl,
                                                const double* etab) {
  double sbb = 0.0;
  int k = 0;
  for (; k + 4 <= n; k += 4) {
    LineVals t[4];
    double og[4], e[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) t[q] = load_line(lt + k + q);
#pragma unroll
    for (int q = 0; q < 4; ++q) og[q] = s_gl[line_row(t[q].idx) * FC];
#pragma unroll
    for (int q = 0; q < 4; ++q)
      e[q] = INRANGE ? exp_tang_inrange(-(t[q].chi * h), etab) : exp_tang(-(t[q].chi * h), etab);
#pragma unroll
    for (int q = 0; q < 4; ++q) sbb = fma(t[q].pg * og[q], e[q], sbb);
  }
  for (; k < n; ++k) {
    const LineVals t = load_line(lt + k);
    const double og = s_gl[line_row(t.idx) * FC];
    const double e = INRANGE ? exp_tang_inrange(-(t.chi * h), etab) : exp_tang(-(t.chi * h), etab);
    sbb = fma(t.pg * og, e, sbb);
  }
  return sbb;
}

// bb_sum_staged for the FS shells of a lane at once (s_gl: the first shell's
// column; the others' are OPAC_CT apart, rows FS * OPAC_CT apart): each line
// record's load and index work serves FS terms.  NL lines per round: FS * NL
// independent exps.
template <bool INRANGE, int FS, int NL>
__device__ __forceinline__ void bb_sum_staged_fs(const LineTerm* lt, int n, const double* h, const double* s_gl,
                                                 const double* etab, double* sbb) {
  constexpr int FC = FS * OPAC_CT;
  double a[FS];
#pragma unroll
  for (int s = 0; s < FS; ++s) a[s] = 0.0;
  int k = 0;
  for (; k + NL <= n; k += NL) {
    LineVals t[NL];
#pragma unroll
    for (int q = 0; q < NL; ++q) t[q] = load_line(lt + k + q);
#pragma unroll
    for (int q = 0; q < NL; ++q) {
      const double* r = s_gl + line_row(t[q].idx) * FC;
#pragma unroll
      for (int s = 0; s < FS; ++s) {
        const double e = INRANGE ? exp_tang_inrange(-(t[q].chi * h[s]), etab) : exp_tang(-(t[q].chi * h[s]), etab);
        a[s] = fma(t[q].pg * r[s * OPAC_CT], e, a[s]);
      }
    }
  }
  for (; k < n; ++k) {
    const LineVals t = load_line(lt + k);
    const double* r = s_gl + line_row(t.idx) * FC;
#pragma unroll
    for (int s = 0; s < FS; ++s) {
      const double e = INRANGE ? exp_tang_inrange(-(t.chi * h[s]), etab) : exp_tang(-(t.chi * h[s]), etab);
      a[s] = fma(t.pg * r[s * OPAC_CT], e, a[s]);
    }
  }
#pragma unroll
  for (int s = 0; s < FS; ++s) sbb[s] = a[s];
}

// Bound-free and free-free of sub-group igs for shell i (h = hc/kT), added to
// cap in the reference's order (after the bound-bound term).
__device__ inline double bf_ff_add(const OpacArgs& A, int i, int igs, double h, double cap) {
  if (!A.nobf) {
    const size_t base = (size_t)(igs - 1) * A.maxact;
    const int n = A.bnnz[igs - 1];
    const double* oci = A.oc + i;
    for (int k = 0; k < n; ++k)  // bfxs * pc_mbarn (the reference's first product) * population
      cap = cap + __ldg(A.xsc + base + k) * oci[(size_t)__ldg(A.bslot + base + k) * A.nc];
  }
  if (!A.noff) {
    const double wl = A.wlsub[igs - 1];
    const double wlinv = 1.0 / wl;
    const double u = h * wlinv;
    const double ru = 10.0 * (log10(u) + 4.0) + 1.0;
    const int iu = !(ru >= 1.0) ? 1 : (ru >= (double)(FF_NU - 1) ? FF_NU - 1 : (int)floor(ru));
    const double du = ru - iu;
    const double help = A.ffc1 * sqrt(h) * (1.0 - exp(-u)) * cube(wl) * A.hlparr[i];
    // sum over elements of z^2 fr gff (ff_sum_kernel), the clamped ones here
    const double* S = A.ffsum + (size_t)i * FF_NU;
    double sg = (1.0 - du) * __ldg(S + iu - 1) + du * __ldg(S + iu);
    for (unsigned m = __ldg(A.ffclamp + i); m; m &= m - 1) {
      const int iz = __ffs(m);
      const int igg = -A.ffigg[(size_t)(iz - 1) * A.nc + i];
      const double dgg = A.ffdgg[(size_t)(iz - 1) * A.nc + i];
      const double* G = A.gff;
      double g = (1.0 - du) * (1.0 - dgg) * G[(iu - 1) + FF_NU * (igg - 1)] +
                 du * (1.0 - dgg) * G[iu + FF_NU * (igg - 1)] +
                 (1.0 - du) * dgg * G[(iu - 1) + FF_NU * igg] + du * dgg * G[iu + FF_NU * igg];
      g = g > 1.0 ? g : 1.0;
      sg = sg + (double)(iz * iz) * A.natomfr[(size_t)(A.nelem + 1) * i + iz] * g;
    }
    cap = cap + help * sg;
  }
  return cap;
}

// 1 - exp(-h / wl(igs)), wl the sub-group's centre: the stimulated-emission
// factor of the bound-bound term (physical_opacity.f:148-149).
__device__ __forceinline__ double bb_expfac(const OpacArgs& A, int igs, double h) {
  const double wa = A.wlsub[igs - 1], wb = A.wlsub[igs];
  const double wl = 0.5 * (wa + wb);
  const double wlinv = 1.0 / wl;
  return 1.0 - exp(-(h * wlinv));
}

// One sub-group igs for shell i: bb, bf and ff in the reference's order.
// etab: the exp table (kExp2Tab) in shared memory; s_gl: the shell's column of
// the block's staged population rows ([line row][FC] in shared memory), or
// null (read grndlev).
template <int FC>
__device__ inline double subgroup_opacity(const OpacArgs& A, int i, const double* s_gl, int igs, bool live,
                                          const double* etab) {
  double cap = 0.0;
  if (!live) return cap;
  const double h = A.hckt[i];
  if (!A.nobb) {
    const int l0 = A.lstart[igs], l1 = A.lstart[igs + 1];
    if (l1 > l0) {
      const double expfac = bb_expfac(A, igs, h);
      // sum over the sub-group's lines of phi gxs ocg exp(-chilw h), times the
      // stimulated-emission factor once (the reference multiplies each term by
      // it; the sum of positive terms differs by rounding only)
      const LineTerm* lt = A.lt + l0;
      const int n = l1 - l0;
      double sbb;
      // h * chimax <= 700: every exp argument -chi h lies in [-700, 0], where
      // exp_tang needs no range check
      const bool inrange = h >= 0.0 && h * A.chimax <= 700.0;
      if (s_gl) {
        // staged populations are clamped at zero, so a term of an unpopulated
        // ion adds +0 (the reference skips it: the same sum)
        sbb = inrange ? bb_sum_staged<true, FC>(lt, n, h, s_gl, etab) : bb_sum_staged<false, FC>(lt, n, h, s_gl, etab);
      } else {
        sbb = 0.0;
        for (int k = 0; k < n; ++k) {
          const LineVals t = load_line(lt + k);
          const double ocg = A.grndlev[(size_t)line_slot(t.idx) * A.nc + i];
          if (ocg <= 0.0) continue;
          sbb = fma(t.pg * ocg, exp_tang(-(t.chi * h), etab), sbb);
        }
      }
      cap = cap + sbb * expfac;
    }
  }
  return bf_ff_add(A, i, igs, h, cap);
}

// Block: FS * OPAC_CT shells x OPAC_GT groups; warp w takes group
// blockIdx.y * OPAC_GT + w + 1, lane l shells base + s OPAC_CT + l, s < FS.
template <int FS>
__global__ void __launch_bounds__(OPAC_GT * 32, 4) opacity_fwd_kernel(const OpacArgs A) {
  constexpr int FC = FS * OPAC_CT;
  __shared__ float tcap[FC][OPAC_GT + 1];
  __shared__ float tem[FC][OPAC_GT + 1];
  __shared__ double tcapd[FC][OPAC_GT + 1];
  __shared__ double etab[kExpTabN];
  extern __shared__ double s_rows[];  // [line row][FC] populations of this block's shells (A.stage_rows)
  exp_table_load(etab);
  const int base = blockIdx.x * FC;
  if (A.stage_rows) {
    for (int k = threadIdx.x; k < A.nlrow * FC; k += blockDim.x) {
      const int ii = base + (k % FC);
      const double v = ii < A.nc ? A.grndlev[(size_t)A.slot_of_lrow[k / FC] * A.nc + ii] : 0.0;
      s_rows[k] = v < 0.0 ? 0.0 : v;  // the reference skips lines with ocg <= 0
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ig = blockIdx.y * OPAC_GT + warp + 1;  // 1-based group
  int ii[FS];
  bool valid[FS], live[FS];
  double cap[FS];
#pragma unroll
  for (int s = 0; s < FS; ++s) {
    ii[s] = base + s * OPAC_CT + lane;  // 0-based shell
    valid[s] = ig <= A.ng && ii[s] < A.nc;
    live[s] = valid[s] && A.mass[ii[s]] > 0.0;
    cap[s] = 0.0;
  }
  if (A.ngs == 1 && A.stage_rows) {
    // both shells' bound-bound sums in one pass over the group's lines
    // (a shell that is not live runs the loop with h = 0 and is discarded)
    double h[FS];
#pragma unroll
    for (int s = 0; s < FS; ++s) h[s] = live[s] ? A.hckt[ii[s]] : 0.0;
    const int l0 = ig <= A.ng ? A.lstart[ig] : 0, l1 = ig <= A.ng ? A.lstart[ig + 1] : 0;
    double sbb[FS];
#pragma unroll
    for (int s = 0; s < FS; ++s) sbb[s] = 0.0;
    if (!A.nobb && l1 > l0) {
      bool inrange = true;
#pragma unroll
      for (int s = 0; s < FS; ++s) inrange = inrange && h[s] >= 0.0 && h[s] * A.chimax <= 700.0;
      constexpr int NL = FS == 2 ? 4 : 2;  // eight exps in flight
      if (inrange)
        bb_sum_staged_fs<true, FS, NL>(A.lt + l0, l1 - l0, h, s_rows + lane, etab, sbb);
      else
        bb_sum_staged_fs<false, FS, NL>(A.lt + l0, l1 - l0, h, s_rows + lane, etab, sbb);
    }
#pragma unroll
    for (int s = 0; s < FS; ++s) {
      if (!live[s]) continue;
      double c = 0.0;
      if (!A.nobb && l1 > l0) c = c + sbb[s] * bb_expfac(A, ig, h[s]);
      cap[s] = bf_ff_add(A, ii[s], ig, h[s], c);
    }
  } else {
#pragma unroll 1
    for (int s = 0; s < FS; ++s) {
      if (!valid[s]) continue;
      const double* s_gl = A.stage_rows ? s_rows + s * OPAC_CT + lane : nullptr;
      if (A.ngs == 1) {
        cap[s] = subgroup_opacity<FC>(A, ii[s], s_gl, ig, live[s], etab);
      } else {
        // collapse subgridding, physical_opacity.f:252-264
        double sp = 0.0, sr = 0.0;
        for (int g = 1; g <= A.ngs; ++g) {
          const double v = subgroup_opacity<FC>(A, ii[s], s_gl, (ig - 1) * A.ngs + g, live[s], etab);
          if (v > 0.0) { sp = sp + v; sr = sr + 1.0 / v; }
        }
        const double help = 1.0 / A.ngs;
        const double capp = sp * help;
        double capr = sr * help;
        if (capr > 0.0) capr = 1.0 / capr;
        cap[s] = (1.0 - A.mix) * capp + A.mix * capr;
      }
    }
  }
#pragma unroll
  for (int s = 0; s < FS; ++s) {
    const int i = ii[s];
    float c32 = (float)cap[s], e32 = 0.f;
    if (live[s]) {
      const double wl = 0.5 * (A.grp_wl[ig] + A.grp_wl[ig - 1]);
      const double B_nu = (wl * wl / pc_c) * planck(wl, A.temp[i]);
      e32 = (float)(0.0 + cap[s] * B_nu);
      int f = 0;
      if (c32 == 0.f) f |= 1;
      if (c32 < 0.f) f |= 2;
      if (c32 != c32) f |= 4;
      if (c32 > FLT_MAX) f |= 8;
      if (f) atomicOr(A.flags, f);
    }
    if (valid[s] && A.cap64) A.cap64[(size_t)(ig - 1) * A.nc + i] = cap[s];
    tcap[s * OPAC_CT + lane][warp] = c32;
    tem[s * OPAC_CT + lane][warp] = e32;
    if (A.capg64) tcapd[s * OPAC_CT + lane][warp] = cap[s];
  }
  __syncthreads();
  // write (ng, ncell): each shell's OPAC_GT consecutive groups together
  for (int t = threadIdx.x; t < FC * OPAC_GT; t += blockDim.x) {
    const int ci = t / OPAC_GT, gj = t % OPAC_GT;
    const int i2 = base + ci, g2 = blockIdx.y * OPAC_GT + gj;
    if (i2 < A.nc && g2 < A.ng) {
      A.cap32[(size_t)i2 * A.ng + g2] = tcap[ci][gj];
      A.emiss32[(size_t)i2 * A.ng + g2] = tem[ci][gj];
      if (A.capg64) A.capg64[(size_t)i2 * A.ng + g2] = tcapd[ci][gj];
    }
  }
}

// ------------------------------------------------------------ analytic opacity
__global__ void analytic_opacity_kernel(int nc, int ng, const double* __restrict__ wlinv,
                                        const double* __restrict__ temp, const double* __restrict__ rho,
                                        int kind, double capcoef, double captpwr, double caprpwr,
                                        double sigcoef, double sigtpwr, double sigrpwr, double ldisp1,
                                        double ldisp2, double* __restrict__ sig, float* __restrict__ cap) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nc * ng) return;
  const int i = (int)(t / ng), ig = (int)(t % ng) + 1;
  const double cc = capcoef * pow(temp[i], captpwr) * pow(rho[i], caprpwr);
  double v;
  if (kind == 1) v = cc;
  else if (kind == 2) {
    const double x1 = pc_hc * wlinv[ig] / pc_kb;
    const double x2 = pc_hc * wlinv[ig - 1] / pc_kb;
    v = 0.5 * cc * (x1 + x2) / sq(x1 * x2);
  } else {
    v = (ig % 2 == 1) ? cc * ldisp1 : cc * ldisp2;
  }
  cap[t] = (float)v;
  if (ig == 1) sig[i] = sigcoef * pow(temp[i], sigtpwr) * pow(rho[i], sigrpwr);
}

// ------------------------------------------------------------ Planck / Rosseland means
// One block per shell; a fixed-shape tree reduction over groups.
__global__ void __launch_bounds__(256) opacity_means_kernel(int nc, int ng, const double* __restrict__ wlinv,
                                                            const double* __restrict__ temp,
                                                            const double* __restrict__ sig,
                                                            const float* __restrict__ cap,
                                                            double* __restrict__ capgrey,
                                                            double* __restrict__ capross) {
  __shared__ double sp[256], sr[256];
  const int i = blockIdx.x;
  const double tinv = 1.0 / temp[i];
  const double hct = hck * tinv;
  const double s = sig ? sig[i] : 0.0;
  double ap = 0.0, ar = 0.0;
  for (int g = threadIdx.x; g < ng; g += blockDim.x) {
    const double c = (double)cap[(size_t)i * ng + g];
    ap = ap + c * specintv_elem(hct, wlinv, g);
    ar = ar + (1.0 / (s + c)) * spectintv_elem(hct, wlinv, g);
  }
  sp[threadIdx.x] = ap;
  sr[threadIdx.x] = ar;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      sp[threadIdx.x] = sp[threadIdx.x] + sp[threadIdx.x + w];
      sr[threadIdx.x] = sr[threadIdx.x] + sr[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    capgrey[i] = sp[0];
    if (capross) capross[i] = 1.0 / sr[0];
  }
}

// ------------------------------------------------------------ adjoint (no reference counterpart)
// specintv_elem and spectintv_elem of group g0 and their d/dT at temperature T
// (hct = hck/T), from one exp of the group's x: the expressions of fplanck and
// fross (so the same values) and of their derivatives in x, which are zero
// where the reference clamps x at 300; spectintv's NaN guard
// (groupmod.f:390-392) gives zero for both.
__device__ inline void spec_weights_dT(double hct, double T, const double* __restrict__ wlinv, int g0, double& w,
                                       double& wr, double& dw, double& dwr) {
  const double x1 = hct * wlinv[g0], x2 = hct * wlinv[g0 + 1];
  const double xm = 0.5 * (x2 + x1), ax = fabs(x2 - x1);
  double fp, fr, dfp, dfr;
  if (xm >= 300.0) {
    fp = fplanck(xm);
    fr = fross(xm);
    dfp = 0.0;
    dfr = 0.0;
  } else {
    const double ex = exp(xm), d = ex - 1.0;
    fp = cube(xm) / d;
    fr = (pow4(xm) * ex) / sq(d);
    dfp = 3.0 * sq(xm) / d - cube(xm) * ex / sq(d);
    const double v = fr * (4.0 / xm + 1.0 - 2.0 * ex / d);
    dfr = v != v ? 0.0 : v;
  }
  w = ftpi4 * ax * fp;
  dw = -(ftpi4 * ax * (fp + xm * dfp)) / T;
  const double sr = ftpi4r * ax * fr;
  const bool bad = sr != sr;  // groupmod.f:390-392
  wr = bad ? 0.0 : sr;
  dwr = bad ? 0.0 : -(ftpi4r * ax * (fr + xm * dfr)) / T;
}

// opacity_planckmean / opacity_rossmean on the FP64 opacity in (ng, ncell) layout.
__global__ void __launch_bounds__(256) opacity_means64_kernel(int nc, int ng, const double* __restrict__ wlinv,
                                                              const double* __restrict__ temp,
                                                              const double* __restrict__ sig,
                                                              const double* __restrict__ cap,
                                                              double* __restrict__ capgrey,
                                                              double* __restrict__ capross) {
  __shared__ double sp[256], sr[256];
  const int i = blockIdx.x;
  const double hct = hck * (1.0 / temp[i]);
  const double s = sig ? sig[i] : 0.0;
  double ap = 0.0, ar = 0.0;
  for (int g = threadIdx.x; g < ng; g += blockDim.x) {
    const double c = cap[(size_t)i * ng + g];
    ap = ap + c * specintv_elem(hct, wlinv, g);
    ar = ar + (1.0 / (s + c)) * spectintv_elem(hct, wlinv, g);
  }
  sp[threadIdx.x] = ap;
  sr[threadIdx.x] = ar;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      sp[threadIdx.x] = sp[threadIdx.x] + sp[threadIdx.x + w];
      sr[threadIdx.x] = sr[threadIdx.x] + sr[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    capgrey[i] = sp[0];
    capross[i] = 1.0 / sr[0];
  }
}

// Adjoint of opacity_means64_kernel: adds to gcap (ng, ncell), gsig and gT.
__global__ void __launch_bounds__(256) means_bwd_kernel(int nc, int ng, const double* __restrict__ wlinv,
                                                        const double* __restrict__ temp,
                                                        const double* __restrict__ sig,
                                                        const double* __restrict__ cap,
                                                        const double* __restrict__ capross,
                                                        const double* __restrict__ ggrey,
                                                        const double* __restrict__ gross, double* __restrict__ gcap,
                                                        double* __restrict__ gsig, double* __restrict__ gT) {
  __shared__ double s1[256], s2[256];
  const int i = blockIdx.x;
  const double T = temp[i], hct = hck * (1.0 / T);
  const double s = sig[i];
  const double ug = ggrey ? ggrey[i] : 0.0;
  const double cr = capross[i];
  const double ur = gross ? gross[i] * cr * cr : 0.0;  // capross = 1/R: d capross = -capross^2 dR
  double asig = 0.0, at = 0.0;
  for (int g = threadIdx.x; g < ng; g += blockDim.x) {
    const double c = cap[(size_t)i * ng + g];
    double w, wr, dw, dwr;
    spec_weights_dT(hct, T, wlinv, g, w, wr, dw, dwr);
    const double inv = 1.0 / (s + c);
    const double dr = wr * inv * inv;  // -dR/dc
    gcap[(size_t)i * ng + g] += ug * w + ur * dr;
    asig = asig + ur * dr;
    at = at + ug * c * dw - ur * inv * dwr;
  }
  s1[threadIdx.x] = asig;
  s2[threadIdx.x] = at;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s1[threadIdx.x] += s1[threadIdx.x + w];
      s2[threadIdx.x] += s2[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    gsig[i] += s1[0];
    gT[i] += s2[0];
  }
}

struct OpacBwd {
  const double* gcap;  // (ng, ncell)
  double* gT;          // (ncell), added to
  double* ggrnd;       // [slot][cell], added to (d cap / d grndlev)
  double* goc;         // [slot][cell], added to (bound-free)
  double* ghlp;        // (ncell), added to (d cap / d hlparr)
  double* gfr;         // (0:nelem, ncell), added to
  double* W;           // [cell][81], added to: free-free table-row weights (null with noff)
};

// The bound-bound part of the adjoint for one (shell, group): adds
// ue * d cap / d grndlev / expfac = ue * pg * exp(-chi h) of every line
// (ue = u * expfac) to dL/d grndlev of its population row: GRED, in global
// memory (acc_l = ggrnd + shell, entry slot * nc: one reduction without
// return per term, coalesced over the warp's shells), else in the block's
// shared accumulator (acc_l = s_grnd + lane, entry row * 32, atomics with
// return).  Global reductions pay when the accumulated array is large (many
// shells x rows: the updates spread over many addresses); on a small one they
// queue on the same addresses, where the shared accumulator wins.  Returns
// the sums over lines of pg exp(-chi h) og (capbb / expfac) and of the same
// times chi (the T-derivative's weight).  Staged populations are clamped at
// zero, so an unpopulated ion's term is +0 as the forward's skip.  Four lines
// per round: independent loads and exps.
template <bool INRANGE, bool GRED>
__device__ __forceinline__ void bb_adjoint_staged(const LineTerm* lt, int n, double h, double ue,
                                                  const double* s_gl, double* acc_l, size_t nc,
                                                  const double* etab, double& sbb, double& schi) {
  int k = 0;
  for (; k + 4 <= n; k += 4) {
    LineVals t[4];
    int r[4];
    double e[4], o[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) t[q] = load_line(lt + k + q);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      r[q] = line_row(t[q].idx) << 5;
      o[q] = s_gl[r[q]];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
      e[q] = t[q].pg * (INRANGE ? exp_tang_inrange(-(t[q].chi * h), etab) : exp_tang(-(t[q].chi * h), etab));
#pragma unroll
    for (int q = 0; q < 4; ++q)
      atomicAdd(acc_l + (GRED ? (size_t)line_slot(t[q].idx) * nc : (size_t)r[q]), ue * e[q]);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double x = e[q] * o[q];
      sbb = sbb + x;
      schi = fma(x, t[q].chi, schi);
    }
  }
  for (; k < n; ++k) {
    const LineVals t = load_line(lt + k);
    const int r = line_row(t.idx) << 5;
    const double e = t.pg * (INRANGE ? exp_tang_inrange(-(t.chi * h), etab) : exp_tang(-(t.chi * h), etab));
    atomicAdd(acc_l + (GRED ? (size_t)line_slot(t.idx) * nc : (size_t)r), ue * e);
    const double x = e * s_gl[r];
    sbb = sbb + x;
    schi = fma(x, t.chi, schi);
  }
}

// Adjoint of subgroup_opacity (ngs = 1): bb and ff in one pass over the lines
// of each group (bf: bf_bwd_kernel); d/d(natomfr) sums gathered per (element,
// shell) in shared memory, d/d(grndlev) as bb_adjoint_staged's GRED says.
template <bool GRED>
__global__ void __launch_bounds__(OPAC_GT * 32, 4) opacity_bwd_kernel(const OpacArgs A, const OpacBwd B) {
  extern __shared__ double sm[];
  const int nrow = A.nlrow;                          // population rows the lines reference
  const int nacc = GRED ? 0 : nrow;                  // shared accumulator rows
  double* s_W = sm;                                  // [81][32] free-free table-row weights
  double* s_grnd = s_W + FF_NU * 32;                 // [line row][32] (not GRED)
  double* s_fr = s_grnd + (size_t)nacc * 32;         // [nelem+1][32]
  double* s_t = s_fr + (size_t)(A.nelem + 1) * 32;   // [warp][32]
  double* s_h = s_t + OPAC_GT * 32;
  double* s_g = s_h + OPAC_GT * 32;                  // [line row][32] populations of this block's shells
  const int ntot = (FF_NU + nacc + A.nelem + 1) * 32;
  __shared__ double etab[kExpTabN];
  exp_table_load(etab);
  for (int k = threadIdx.x; k < ntot; k += blockDim.x) sm[k] = 0.0;
  for (int k = threadIdx.x; k < nrow * 32; k += blockDim.x) {
    const int ii = blockIdx.x * OPAC_CT + (k & 31);
    const double v = ii < A.nc ? A.grndlev[(size_t)A.slot_of_lrow[k >> 5] * A.nc + ii] : 0.0;
    s_g[k] = v < 0.0 ? 0.0 : v;  // the forward skips lines with ocg <= 0: a zero term
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ig = blockIdx.y * OPAC_GT + warp + 1;
  const int i = blockIdx.x * OPAC_CT + lane;
  const bool live = ig <= A.ng && i < A.nc && A.mass[i] > 0.0;
  double gt = 0.0, gh = 0.0;
  const double u = live ? B.gcap[(size_t)i * A.ng + (ig - 1)] : 0.0;
  if (u != 0.0) {
    const double h = A.hckt[i], T = A.temp[i];
    if (!A.nobb) {
      const int l0 = A.lstart[ig], l1 = A.lstart[ig + 1];
      if (l1 > l0) {
        const double wa = A.wlsub[ig - 1], wb = A.wlsub[ig];
        const double wl = 0.5 * (wa + wb);
        const double wlinv = 1.0 / wl;
        const double eh = exp(-(h * wlinv));
        const double expfac = 1.0 - eh;
        double sbb = 0.0, schi = 0.0;
        const double ue = u * expfac;
        const bool inrange = h >= 0.0 && h * A.chimax <= 700.0;  // as in the forward
        double* acc_l = GRED ? B.ggrnd + i : s_grnd + lane;
        if (inrange)
          bb_adjoint_staged<true, GRED>(A.lt + l0, l1 - l0, h, ue, s_g + lane, acc_l, A.nc, etab, sbb, schi);
        else
          bb_adjoint_staged<false, GRED>(A.lt + l0, l1 - l0, h, ue, s_g + lane, acc_l, A.nc, etab, sbb, schi);
        const double capbb = sbb * expfac;
        schi = schi * expfac;
        // h = hc/kT: d exp(-chi h)/dT = chi h/T exp(..), d expfac/dT = -(h/T) wlinv eh
        gt = gt + u * ((h / T) * schi - capbb * (h / T) * wlinv * eh / expfac);
      }
    }
    // bound-free: bf_bwd_kernel
    if (!A.noff) {
      const double wl = A.wlsub[ig - 1];
      const double wlinv = 1.0 / wl;
      const double uu = h * wlinv;
      const double ru = 10.0 * (log10(uu) + 4.0) + 1.0;
      const int iu = !(ru >= 1.0) ? 1 : (ru >= (double)(FF_NU - 1) ? FF_NU - 1 : (int)floor(ru));
      const double du = ru - iu;
      const double eu = exp(-uu);
      const double hn = A.ffc1 * sqrt(h) * (1.0 - eu) * cube(wl);
      const double help = hn * A.hlparr[i];
      const double dlnhelp = -0.5 / T - eu * uu / (T * (1.0 - eu));
      const double ln10 = 2.302585092994045684;
      const double dru = -10.0 / (ln10 * T), drgg = -5.0 / (ln10 * T);  // table coordinates vs T
      // this group's weights of table rows iu - 1 and iu, for d cap / d fr of
      // the unclamped elements (ff_fr_bwd_kernel)
      atomicAdd(&s_W[(iu - 1) * 32 + lane], u * help * (1.0 - du));
      atomicAdd(&s_W[iu * 32 + lane], u * help * du);
      // unclamped elements from the shell's sums over elements (ff_sum_kernel):
      // S = sum z^2 fr gff, dS/dT through the table row (du) and column (dgg)
      const double* Sv = A.ffsum + (size_t)i * FF_NU;
      const double* Dv = A.ffdsum + (size_t)i * FF_NU;
      const double s0 = Sv[iu - 1], s1 = Sv[iu];
      double S = (1.0 - du) * s0 + du * s1;
      double dS = (s1 - s0) * dru + ((1.0 - du) * Dv[iu - 1] + du * Dv[iu]) * drgg;
      // elements under the gff >= 1 clamp, one by one
      const double* nfr = A.natomfr + (size_t)(A.nelem + 1) * i;
      for (unsigned m = A.ffclamp_all[i]; m; m &= m - 1) {
        const int iz = __ffs(m);
        const double fr = nfr[iz];
        const int igg = -A.ffigg[(size_t)(iz - 1) * A.nc + i];
        const double dgg = A.ffdgg[(size_t)(iz - 1) * A.nc + i];
        const double* G = A.gff;
        const double g00 = G[(iu - 1) + FF_NU * (igg - 1)], g10 = G[iu + FF_NU * (igg - 1)];
        const double g01 = G[(iu - 1) + FF_NU * igg], g11 = G[iu + FF_NU * igg];
        const double graw = (1.0 - du) * (1.0 - dgg) * g00 + du * (1.0 - dgg) * g10 + (1.0 - du) * dgg * g01 +
                            du * dgg * g11;
        const bool flat = graw < 1.0;
        const double g = flat ? 1.0 : graw;
        const double dg = flat ? 0.0
                               : ((1.0 - dgg) * (g10 - g00) + dgg * (g11 - g01)) * dru +
                                     ((1.0 - du) * (g01 - g00) + du * (g11 - g10)) * drgg;
        const double w = (double)(iz * iz);
        atomicAdd(&s_fr[iz * 32 + lane], u * help * g * w);
        if (fr == 0.0) continue;
        S = S + g * w * fr;
        dS = dS + dg * w * fr;
      }
      gh = gh + u * hn * S;
      gt = gt + u * (help * S * dlnhelp + help * dS);
    }
  }
  s_t[warp * 32 + lane] = gt;
  s_h[warp * 32 + lane] = gh;
  __syncthreads();
  if (warp == 0 && i < A.nc) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < OPAC_GT; ++w) {
      a += s_t[w * 32 + lane];
      b += s_h[w * 32 + lane];
    }
    if (a != 0.0) atomicAdd(&B.gT[i], a);
    if (b != 0.0) atomicAdd(&B.ghlp[i], b);
  }
  for (int k = threadIdx.x; k < ntot; k += blockDim.x) {
    const double v = sm[k];
    const int row = k >> 5, c = blockIdx.x * OPAC_CT + (k & 31);
    if (v == 0.0 || c >= A.nc) continue;
    if (row < FF_NU) atomicAdd(&B.W[(size_t)c * FF_NU + row], v);
    else if (row < FF_NU + nacc) atomicAdd(&B.ggrnd[(size_t)A.slot_of_lrow[row - FF_NU] * A.nc + c], v);
    else atomicAdd(&B.gfr[(size_t)c * (A.nelem + 1) + (row - FF_NU - nacc)], v);
  }
}

// Bound-free part of the adjoint (physical_opacity.f:163-195, ngs = 1):
// d cap(g, i) / d oc(slot, i) = xs(g, slot) mbarn, so
// goc(act_slot(a), i) += mbarn sum_g gcap(g, i) xs(g, a) over the active slots a
// -- a product of the (shell, group) gradient with the (group, slot) table.
// Tiled like a matrix product: a block computes 32 shells x 32 slots, staging
// 32 groups of both operands in shared memory per round; thread (tx, ty)
// holds shell tx and slots ty, ty + 8, ty + 16, ty + 24.  Runs after
// opacity_bwd_kernel and before opac_cell_bwd_kernel (one writer per entry).
constexpr int BFB_T = 32;
// shells from which the forward takes four shells per lane
constexpr int kFwdFourShellsMin = 2048;
// d cap(g, i) / d fr(z, i) = help(g, i) z^2 gff_z(g, i) for the elements
// without the gff >= 1 clamp, where gff_z = (1 - du_g) Gz[iu_g - 1] + du_g
// Gz[iu_g] is linear in the table-row weights: sum_g u_g help_g gff_z =
// sum_j W[j] Gz[j] with W[j] the row weights of all groups, weighted by
// u_g help_g (u = dL/dcap).  opacity_bwd_kernel gathers W per block in shared
// memory and adds its nonzero entries (a block's eight groups touch a few rows
// per shell), ff_fr_bwd_kernel adds
// z^2 sum_j W[j] Gz[j] to gfr (after opacity_bwd_kernel, which adds the
// clamped elements).
__global__ void ff_fr_bwd_kernel(const OpacArgs A, const double* __restrict__ W, double* __restrict__ gfr) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)A.nc * A.nelem) return;
  const int i = (int)(t / A.nelem), iz = (int)(t % A.nelem) + 1;
  const int igg = A.ffigg[(size_t)(iz - 1) * A.nc + i];
  if (igg < 0) return;  // clamped: opacity_bwd_kernel
  const double dgg = A.ffdgg[(size_t)(iz - 1) * A.nc + i];
  const double* G = A.gff;
  const double* w = W + (size_t)i * FF_NU;
  double acc = 0.0;
  for (int j = 0; j < FF_NU; ++j) acc = acc + w[j] * ((1.0 - dgg) * G[j + FF_NU * (igg - 1)] + dgg * G[j + FF_NU * igg]);
  gfr[(size_t)i * (A.nelem + 1) + iz] += (double)(iz * iz) * acc;
}

// population rows x shells from which the adjoint accumulates d/d(population)
// in global memory: measured on B200, shared accumulators won at 40 rows x 256
// shells and global reductions at 40 rows x 4096 shells
constexpr size_t kBwdGlobalAccMin = 32768;
__global__ void __launch_bounds__(BFB_T * 8) bf_bwd_kernel(const OpacArgs A, const OpacBwd B) {
  __shared__ double su[BFB_T][BFB_T + 1];  // [shell][group]
  __shared__ double sx[BFB_T][BFB_T + 1];  // [group][slot]
  const int nact = *A.pnact;
  const int a0 = blockIdx.y * BFB_T;
  if (a0 >= nact) return;  // uniform over the block
  const int i0 = blockIdx.x * BFB_T;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int g0 = 0; g0 < A.ng; g0 += BFB_T) {
    // the cross sections first: most (group, slot) tiles lie beyond the slots'
    // ionisation edges, all zero, and are skipped (the forward skips xs = 0)
    bool nz = false;
    for (int k = threadIdx.x; k < BFB_T * BFB_T; k += blockDim.x) {
      const int r = k >> 5, q = k & 31;  // sx: group r, slot q
      const int gr = g0 + r, a = a0 + q;
      const double x = (gr < A.ng && a < nact) ? A.xstab[(size_t)gr * A.maxact + a] : 0.0;
      sx[r][q] = x;
      nz = nz || x != 0.0;
    }
    if (!__syncthreads_or(nz)) continue;  // block-uniform
    for (int k = threadIdx.x; k < BFB_T * BFB_T; k += blockDim.x) {
      const int r = k >> 5, q = k & 31;  // su: shell r, group q (coalesced over groups)
      const int ii = i0 + r, g = g0 + q;
      su[r][q] = (ii < A.nc && g < A.ng) ? B.gcap[(size_t)ii * A.ng + g] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int q = 0; q < BFB_T; ++q) {
      const double u = su[tx][q];
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[j] = acc[j] + u * sx[q][ty + 8 * j];
    }
    __syncthreads();
  }
  const int i = i0 + tx;
  if (i >= A.nc || !(A.mass[i] > 0.0)) return;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int a = a0 + ty + 8 * j;
    if (a < nact && acc[j] != 0.0) B.goc[(size_t)A.act_slot[a] * A.nc + i] += acc[j];  // xstab holds * pc_mbarn
  }
}

// Adjoint of opac_cell_prep_kernel: grndlev = oc ginv, hlparr = (natom/vol)^2
// nelec, gas_sig = cthomson nelec natom / vol.
__global__ void opac_cell_bwd_kernel(int nc, int nelem, int nst, const int32_t* __restrict__ ion_ni,
                                     const double* __restrict__ natom, const double* __restrict__ nelec,
                                     const double* __restrict__ vol, const double* __restrict__ mass,
                                     const double* __restrict__ ginv, int nothmson,
                                     const double* __restrict__ ggrnd, const double* __restrict__ ghlp,
                                     const double* __restrict__ gsig, double* __restrict__ goc,
                                     double* __restrict__ gnelec, double* __restrict__ gnatom) {
  // one thread per (shell i, element iz = blockIdx.y + 1); element 1's threads
  // also write the shell's scalars
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nc) return;
  if (!(mass[i] > 0.0)) {
    if (blockIdx.y == 0) {
      gnelec[i] = 0.0;
      gnatom[i] = 0.0;
    }
    return;
  }
  {
    const int iz = blockIdx.y + 1;
    const int lim = min(iz, ion_ni[iz - 1] - 1);
    for (int ii = 1; ii <= lim && ii <= nst; ++ii) {
      const size_t k = ((size_t)(iz - 1) * nst + (ii - 1)) * nc + i;
      goc[k] += ggrnd[k] * ginv[k];
    }
  }
  if (blockIdx.y != 0) return;
  const double nd = natom[i] / vol[i];
  double gne = ghlp[i] * nd * nd;
  double gna = ghlp[i] * 2.0 * nd * nelec[i] / vol[i];
  if (!nothmson) {
    gne += gsig[i] * cthomson * natom[i] / vol[i];
    gna += gsig[i] * cthomson * nelec[i] / vol[i];
  }
  gnelec[i] = gne;
  gnatom[i] = gna;
}

}  // namespace

// ============================================================ launchers
// One launch of opacity_fwd_kernel on the stream.  Shells per lane: 4 on large
// grids (each line record serves four terms; measured on B200 at 4096 shells:
// 11.2 against 11.7 ms), 2 where four would leave too few blocks for the SMs
// (256 shells: 0.39 against 0.41 ms) or too many staged rows.  The block's
// population rows are staged in shared memory up to 80 KB of them (beyond,
// the kernel reads grndlev); the kernel's dynamic limit is raised on the
// device before its first staged launch (with its static arrays a block
// passes the default 48 KB from about 77 rows at 2 shells per lane).
static int launch_fwd(slg_ctx* ctx, OpacArgs& A) {
  const size_t rows4 = sizeof(double) * 4 * OPAC_CT * (size_t)A.nlrow;
  const bool four = A.nc >= kFwdFourShellsMin && (A.nobb || A.nlrow == 0 || rows4 <= 80 * 1024);
  const int fs = four ? 4 : 2;
  const size_t b = sizeof(double) * fs * OPAC_CT * (size_t)A.nlrow;
  A.stage_rows = (!A.nobb && A.nlrow > 0 && b <= 80 * 1024) ? 1 : 0;
  const size_t shm = A.stage_rows ? b : 0;
  static unsigned raised[2] = {0, 0};  // per device and form
  const dim3 grid((A.nc + fs * OPAC_CT - 1) / (fs * OPAC_CT), (A.ng + OPAC_GT - 1) / OPAC_GT);
  if (four) {
    raise_smem_limit(raised[1], ctx->device, opacity_fwd_kernel<4>, 80 * 1024);
    opacity_fwd_kernel<4><<<grid, OPAC_GT * 32, shm, ctx->stream>>>(A);
  } else {
    raise_smem_limit(raised[0], ctx->device, opacity_fwd_kernel<2>, 80 * 1024);
    opacity_fwd_kernel<2><<<grid, OPAC_GT * 32, shm, ctx->stream>>>(A);
  }
  return cuda_check(ctx, cudaGetLastError(), "opacity_fwd launch");
}

// Everything the opacity kernels read, queued on the stream: sub-group edges,
// the line binning, per-cell terms (and gas_sig) and the bound-free table.
static int opacity_prepare(slg_ctx* ctx, const slg_gas* gas, const slg_opacity_flags* flags, double* gas_sig,
                           OpacArgs& A) {
  const int nc = ctx->nx, ng = ctx->ng;
  const int ngs = flags->ngs < 1 ? 1 : flags->ngs;
  const int ngsub = ng * ngs;
  const int nelem = ctx->nelem, nst = ctx->nstage;
  const int nslot = nelem * nst;
  cudaStream_t st = ctx->stream;
  if (nelem <= 0) return set_error(ctx, SLG_ERR_STATE, "atomic data not set");
  const int nedge = ngsub + 1, nedge_pad = (nedge + 1) & ~1;
  double* d_wlsub = (double*)scratch(ctx, 0, sizeof(double) * nedge_pad);
  unsigned int* d_counts = (unsigned int*)scratch(ctx, 1, sizeof(unsigned int) * (nedge + 2));
  int* d_lstart = (int*)scratch(ctx, 2, sizeof(int) * (nedge + 3));
  int* d_flags = (int*)scratch(ctx, 3, sizeof(int) * 4);
  double* d_hckt = (double*)scratch(ctx, 4, sizeof(double) * nc);
  double* d_hlp = (double*)scratch(ctx, 5, sizeof(double) * nc);
  double* d_grnd = (double*)scratch(ctx, 6, sizeof(double) * (size_t)nc * nslot);
  int* d_ffigg = (int*)scratch(ctx, 7, sizeof(int) * (size_t)nc * nelem);
  double* d_ffdgg = (double*)scratch(ctx, 8, sizeof(double) * (size_t)nc * nelem);
  int* d_active = (int*)scratch(ctx, 9, sizeof(int) * (nslot + 1));
  int16_t* d_act = (int16_t*)scratch(ctx, 10, sizeof(int16_t) * nslot);
  double* d_xs = (double*)scratch(ctx, 11, sizeof(double) * (size_t)ngsub * nslot);
  if (!d_wlsub || !d_counts || !d_lstart || !d_flags || !d_hckt || !d_hlp || !d_grnd || !d_ffigg ||
      !d_ffdgg || !d_active || !d_act || !d_xs)
    return SLG_ERR_OOM;
  int* d_nact = d_active + nslot;
  cudaMemsetAsync(d_counts, 0, sizeof(unsigned int) * (nedge + 2), st);
  cudaMemsetAsync(d_flags, 0, sizeof(int) * 4, st);
  cudaMemsetAsync(d_active, 0, sizeof(int) * (nslot + 1), st);
  wlsub_kernel<<<(nedge_pad + 255) / 256, 256, 0, st>>>(ng, ngs, nedge_pad, ctx->d_wl, d_wlsub);
  const bool do_bb = ctx->nline > 0 && !flags->nobb;
  LineTerm* d_lt = nullptr;
  if (do_bb) {
    const size_t shm = 16 + sizeof(double) * nedge_pad + sizeof(unsigned int) * (nedge + 1);
    if (shm > 220 * 1024)
      return set_error(ctx, SLG_ERR_ARG, "too many sub-groups for line binning (%d)", ngsub);
    static unsigned raised = 0;  // per device; no attribute calls on repeated launches
    raise_smem_limit(raised, ctx->device, bin_lines_kernel, 220 * 1024);
    const int64_t per_block = 256 * 8;
    const int nb = (int)((ctx->nline + per_block - 1) / per_block);
    bin_lines_kernel<<<nb, 256, shm, st>>>(ctx->d_bb, ctx->nline, d_wlsub, nedge, nedge_pad, d_counts,
                                           d_flags);
    scan_counts_kernel<<<1, 1024, 0, st>>>(d_counts, nedge + 1, d_lstart);
    d_lt = (LineTerm*)scratch(ctx, 84, sizeof(LineTerm) * (size_t)ctx->nline);
    if (!d_lt) return SLG_ERR_OOM;
    decode_lines_kernel<<<(unsigned)((ctx->nline + 255) / 256), 256, 0, st>>>(
        ctx->d_bb, ctx->nline, d_lstart, ngsub, d_wlsub, nst, ctx->d_lrow_of_slot, d_lt);
  } else {
    cudaMemsetAsync(d_lstart, 0, sizeof(int) * (nedge + 3), st);
  }
  opac_cell_prep_kernel<<<dim3((nc + 127) / 128, nelem), 128, 0, st>>>(
      nc, nelem, nst, ctx->d_ion_ni, gas->temp, gas->natom, gas->nelec, gas->vol, gas->mass, gas->oc,
      gas->ginv, flags->nothmson, d_hckt, gas_sig, d_hlp, d_grnd, d_ffigg, d_ffdgg);
  double *d_ffsum = nullptr, *d_ffdsum = nullptr;
  unsigned* d_ffclamp = nullptr;
  if (!flags->noff && ctx->d_gff) {
    d_ffsum = (double*)scratch(ctx, 88, sizeof(double) * 2 * (size_t)nc * FF_NU);
    d_ffclamp = (unsigned*)scratch(ctx, 89, sizeof(unsigned) * 2 * (size_t)nc);
    if (!d_ffsum || !d_ffclamp) return SLG_ERR_OOM;
    d_ffdsum = d_ffsum + (size_t)nc * FF_NU;
    const int64_t nt = (int64_t)nc * FF_NU;
    ff_sum_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(nc, nelem, gas->natomfr, d_ffigg, d_ffdgg,
                                                                ctx->d_gff, d_ffsum, d_ffdsum, d_ffclamp,
                                                                d_ffclamp + nc);
  }
  const bool do_bf = !flags->nobf;
  double* d_xsc = nullptr;
  int *d_bslot = nullptr, *d_bnnz = nullptr;
  if (do_bf) {
    dim3 ga((nc + 255) / 256 < 8 ? (nc + 255) / 256 : 8, nslot);
    ion_active_kernel<<<ga, 256, 0, st>>>(nc, gas->oc, d_active);
    ion_compact_kernel<<<1, 32, 0, st>>>(nelem, nst, ctx->d_ion_ni, d_active, d_act, d_nact);
    const int64_t nt = (int64_t)ngsub * nslot;
    bf_table_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(ngsub, nslot, d_nact, d_act, nst, d_wlsub,
                                                                  ctx->d_ph1, ctx->d_ph2, d_xs);
    d_xsc = (double*)scratch(ctx, 85, sizeof(double) * (size_t)ngsub * nslot);
    d_bslot = (int*)scratch(ctx, 86, sizeof(int) * (size_t)ngsub * nslot);
    d_bnnz = (int*)scratch(ctx, 87, sizeof(int) * (size_t)ngsub);
    if (!d_xsc || !d_bslot || !d_bnnz) return SLG_ERR_OOM;
    bf_compact_kernel<<<(ngsub + 7) / 8, 256, 0, st>>>(ngsub, nslot, d_nact, d_act, d_xs, d_xsc, d_bslot, d_bnnz);
  }
  A.nc = nc; A.ng = ng; A.ngs = ngs; A.ngsub = ngsub; A.nelem = nelem; A.nst = nst; A.maxact = nslot;
  A.pnact = d_nact;
  A.nobb = !do_bb; A.nobf = !do_bf; A.noff = flags->noff;
  A.mix = flags->opacmixrossel;
  A.wlsub = d_wlsub; A.grp_wl = ctx->d_wl; A.lstart = d_lstart; A.bb = ctx->d_bb;
  A.lt = d_lt; A.chimax = ctx->line_chimax; A.slot_of_lrow = ctx->d_slot_of_lrow; A.nlrow = ctx->nlrow;
  A.grndlev = d_grnd; A.oc = gas->oc; A.act_slot = d_act; A.xstab = d_xs;
  A.xsc = d_xsc; A.bslot = d_bslot; A.bnnz = d_bnnz;
  A.hckt = d_hckt; A.hlparr = d_hlp; A.mass = gas->mass; A.natomfr = gas->natomfr; A.temp = gas->temp;
  A.ffigg = d_ffigg; A.ffdgg = d_ffdgg; A.gff = ctx->d_gff;
  A.ffsum = d_ffsum; A.ffdsum = d_ffdsum; A.ffclamp = d_ffclamp;
  A.ffclamp_all = d_ffclamp ? d_ffclamp + nc : nullptr;
  A.ffc1 = ff_c1a * sqrt(ff_c1b);
  A.cap32 = nullptr; A.emiss32 = nullptr; A.cap64 = nullptr; A.capg64 = nullptr; A.flags = d_flags;
  if (!ctx->d_gff && !A.noff) return set_error(ctx, SLG_ERR_STATE, "free-free table not set");
  return SLG_OK;
}

int launch_physical_opacity(slg_ctx* ctx, const slg_gas* gas, const slg_opacity_flags* flags,
                            double* gas_sig, float* gas_cap, float* gas_emiss, double* cap64) {
  OpacArgs A;
  const int rc = opacity_prepare(ctx, gas, flags, gas_sig, A);
  if (rc) return rc;
  A.cap32 = gas_cap; A.emiss32 = gas_emiss; A.cap64 = cap64;
  return launch_fwd(ctx, A);
}

// Physical opacity (ngs = 1) with the FP64 result in gas_cap's (ng, ncell)
// layout; gas_cap/gas_emiss (float) are written as well.
int launch_physical_opacity64(slg_ctx* ctx, const slg_gas* gas, double* gas_sig, double* capg64, float* gas_cap,
                              float* gas_emiss) {
  slg_opacity_flags fl{0, 0, 0, 0, 1, 0.0};
  OpacArgs A;
  const int rc = opacity_prepare(ctx, gas, &fl, gas_sig, A);
  if (rc) return rc;
  A.cap32 = gas_cap; A.emiss32 = gas_emiss; A.capg64 = capg64;
  return launch_fwd(ctx, A);
}

int launch_opacity_means64(slg_ctx* ctx, const double* temp, const double* sig, const double* cap,
                           double* capgrey, double* capross) {
  opacity_means64_kernel<<<ctx->nx, 256, 0, ctx->stream>>>(ctx->nx, ctx->ng, ctx->d_wlinv, temp, sig, cap,
                                                          capgrey, capross);
  return cuda_check(ctx, cudaGetLastError(), "opacity_means64 launch");
}

int launch_means_bwd(slg_ctx* ctx, const double* temp, const double* sig, const double* cap, const double* capross,
                     const double* ggrey, const double* gross, double* gcap, double* gsig, double* gT) {
  means_bwd_kernel<<<ctx->nx, 256, 0, ctx->stream>>>(ctx->nx, ctx->ng, ctx->d_wlinv, temp, sig, cap, capross, ggrey,
                                                    gross, gcap, gsig, gT);
  return cuda_check(ctx, cudaGetLastError(), "means adjoint launch");
}

// Adjoint of launch_physical_opacity64 for gcap (ng, ncell) and gsig: adds
// dL/dT to gT and writes dL/d(oc, nelec, natom, natomfr) (goc [slot][cell],
// gnelec, gnatom, gfr (0:nelem, ncell)).  work: nslot*ncell + ncell doubles.
int launch_opacity_bwd(slg_ctx* ctx, const slg_gas* gas, const double* gcap, const double* gsig, double* gT,
                       double* goc, double* gnelec, double* gnatom, double* gfr, double* sig_work, double* work) {
  slg_opacity_flags fl{0, 0, 0, 0, 1, 0.0};
  OpacArgs A;
  int rc = opacity_prepare(ctx, gas, &fl, sig_work, A);
  if (rc) return rc;
  const int nc = ctx->nx, nslot = A.nelem * A.nst;
  double* ggrnd = work;
  double* ghlp = work + (size_t)nslot * nc;
  cudaStream_t st = ctx->stream;
  cudaMemsetAsync(ggrnd, 0, sizeof(double) * ((size_t)nslot * nc + nc), st);
  cudaMemsetAsync(goc, 0, sizeof(double) * (size_t)nslot * nc, st);
  cudaMemsetAsync(gfr, 0, sizeof(double) * (size_t)nc * (A.nelem + 1), st);
  double* W = nullptr;
  if (!A.noff) {
    W = (double*)scratch(ctx, 90, sizeof(double) * ((size_t)nc * FF_NU + 1));
    if (!W) return SLG_ERR_OOM;
    cudaMemsetAsync(W, 0, sizeof(double) * ((size_t)nc * FF_NU + 1), st);
  }
  OpacBwd B{gcap, gT, ggrnd, goc, ghlp, gfr, W};
  // d/d(population) accumulated in global memory when that array (rows x
  // shells) is large, in shared memory otherwise (bb_adjoint_staged)
  // (and where the shared accumulators would not fit in a block's shared memory)
  auto bwd_smem = [&](bool g) {
    return sizeof(double) * ((size_t)(FF_NU + (g ? 1 : 2) * A.nlrow + A.nelem + 1) * 32 + 2 * OPAC_GT * 32);
  };
  const bool gred = (size_t)A.nlrow * nc >= kBwdGlobalAccMin || bwd_smem(false) > 200 * 1024;
  const size_t shm = bwd_smem(gred);
  if (shm > 200 * 1024) return set_error(ctx, SLG_ERR_ARG, "opacity adjoint: too many ion slots (%d)", A.nlrow);
  static unsigned raised[2] = {0, 0};  // per device and form (with the static table, before 48 KB)
  if (gred) raise_smem_limit(raised[1], ctx->device, opacity_bwd_kernel<true>, 200 * 1024);
  else raise_smem_limit(raised[0], ctx->device, opacity_bwd_kernel<false>, 200 * 1024);
  dim3 grid((nc + OPAC_CT - 1) / OPAC_CT, (A.ng + OPAC_GT - 1) / OPAC_GT);
  if (gred)
    opacity_bwd_kernel<true><<<grid, OPAC_GT * 32, shm, st>>>(A, B);
  else
    opacity_bwd_kernel<false><<<grid, OPAC_GT * 32, shm, st>>>(A, B);
  if (!A.noff) {
    const int64_t nf = (int64_t)nc * A.nelem;
    ff_fr_bwd_kernel<<<(unsigned)((nf + 255) / 256), 256, 0, st>>>(A, W, gfr);
  }
  if (!A.nobf) {
    const dim3 bgrid((nc + BFB_T - 1) / BFB_T, (A.maxact + BFB_T - 1) / BFB_T);
    bf_bwd_kernel<<<bgrid, BFB_T * 8, 0, st>>>(A, B);
  }
  opac_cell_bwd_kernel<<<dim3((nc + 127) / 128, A.nelem), 128, 0, st>>>(nc, A.nelem, A.nst, ctx->d_ion_ni, gas->natom, gas->nelec,
                                                         gas->vol, gas->mass, gas->ginv, 0, ggrnd, ghlp, gsig, goc,
                                                         gnelec, gnatom);
  return cuda_check(ctx, cudaGetLastError(), "opacity adjoint launch");
}

// Sanity bitmask of physical_opacity.f:282-291 (word 0) and line-binning
// errors (word 1: 1 unsorted lines, 2 shared-memory staging time-out).
int opacity_flags(slg_ctx* ctx, int32_t* sanity, int32_t* binning) {
  int* d_flags = (int*)scratch(ctx, 3, sizeof(int) * 4);
  int h[2] = {0, 0};
  int rc = cuda_check(ctx, cudaMemcpyAsync(h, d_flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream),
                      "flags download");
  if (rc) return rc;
  if ((rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "flags sync"))) return rc;
  if (sanity) *sanity = h[0];
  if (binning) *binning = h[1];
  return SLG_OK;
}

int launch_analytic_opacity(slg_ctx* ctx, const double* temp, const double* rho, int kind,
                            const double* c, double* gas_sig, float* gas_cap) {
  const int64_t nt = (int64_t)ctx->nx * ctx->ng;
  analytic_opacity_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, ctx->stream>>>(
      ctx->nx, ctx->ng, ctx->d_wlinv, temp, rho, kind, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7],
      gas_sig, gas_cap);
  return cuda_check(ctx, cudaGetLastError(), "analytic_opacity launch");
}

int launch_opacity_means(slg_ctx* ctx, const double* temp, const double* sig, const float* cap,
                         double* capgrey, double* capross) {
  opacity_means_kernel<<<ctx->nx, 256, 0, ctx->stream>>>(ctx->nx, ctx->ng, ctx->d_wlinv, temp, sig, cap,
                                                        capgrey, capross);
  return cuda_check(ctx, cudaGetLastError(), "opacity_means launch");
}

}  // namespace slg
