// transport.cu -- the 1-D spherical IMC/DDMC particle loop (FP64 form) and the
// flux / source tallies, for sm_100a.
//
// Reference: particle_advance.f90:4-327, fluxtally.f:3-61, sourcetally.f:3-48.
//
// Layout and scheduling:
//  * A persistent grid (a multiple of the SM count) processes particles one
//    event per loop iteration.  A lane whose particle has finished takes the
//    next slot from a global counter; the lanes of a warp that need work in
//    the same iteration share one atomicAdd (warp-aggregated).  This keeps
//    lanes busy while long DDMC random walks finish (lifetimes differ by
//    orders of magnitude).
//  * Particle state lives in registers for the whole flight; the 64-byte
//    packet is read and written once with 16-byte vector accesses.
//  * grd_tally / grd_jrad are accumulated in registers while the (cell,group)
//    of consecutive events is unchanged and flushed with FP64 atomics;
//    counters go through shared-memory atomics and one global atomic per block.
//  * Random numbers: one Philox4x32-10 stream per particle (shared with the
//    oracle), so event sequences can be compared particle by particle.
#include <cuda_runtime.h>
#include <cfloat>
#include "slg_device.cuh"
#include "slg_internal.h"
#include "transport_impl.cuh"

namespace slg {
namespace {

constexpr int TRN_BLOCK = 128;

__device__ inline void load_packet(const slg_packet* p, double& x, double& y, double& z, double& mu,
                                   double& om, double& e, double& e0, double& wl) {
  const double2* q = reinterpret_cast<const double2*>(p);
  const double2 a = q[0], b = q[1], c = q[2], d = q[3];
  x = a.x; y = a.y; z = b.x; mu = b.y; om = c.x; e = c.y; e0 = d.x; wl = d.y;
}
// an escaped particle's slot: x = huge, and its lab-frame mu, e, e0, wl
// (y, z and om are never changed in the slot)
__device__ inline void store_flux_packet(slg_packet* p, double mu, double e, double e0, double wl) {
  p->x = DBL_MAX;
  p->mu = mu;
  p->e = e;
  reinterpret_cast<double2*>(p)[3] = make_double2(e0, wl);
}

// MINB = minimum resident blocks per SM requested from the register
// allocator: 1 -> up to 255 registers (the compiler settles on 128),
// 5 -> 96, 6 -> 80, 8 -> 64 registers with some spilling.  The autotuner
// (slg_autotune_transport) picks the fastest on the caller's workload.
// MODELS: the slots belong to several independent models (slg_set_models);
// each particle finds its model once, draws from its model's random key with
// the model-local slot as counter (as the model would alone), and tallies
// into its model's cells.
template <bool TRACE, int MINB, bool MODELS = false>
__global__ void __launch_bounds__(TRN_BLOCK, MINB) particle_advance_kernel(const TrnArgs A) {
  __shared__ unsigned long long s_cnt[20];
  __shared__ double s_sum[3];
  if (threadIdx.x < 20) s_cnt[threadIdx.x] = 0ull;
  if (threadIdx.x < 3) s_sum[threadIdx.x] = 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  // counters are kept per particle in 32 bits (DDMC steps, method swaps; the
  // IMC steps are istep - nd_p) and added to the block's shared counters when
  // the particle ends, so few registers carry them through the loop
  double evelo = 0.0;
  unsigned nd_p = 0, nsw_p = 0;
  // current particle
  long long ip = -1;
  bool have = false;
  Ptcl p;
  PhiloxStream rng;
  // replays of a captured graph draw from counter word 3 = stream | replay << 2
  const uint32_t sw = A.epoch ? (uint32_t)(*A.epoch << 2) : 0u;
  int istep = 0;
  uint64_t h = 0;
  // the current particle's model: shells, first cell, first shell edge
  int vnx = A.nx, vco = 0, vxo = 0;
  // register caches of the tallies
  int t_ic = 0;
  double t_acc = 0.0;
  int j_ic = 0, j_ig = 0;
  double j_acc = 0.0;
  bool queue_done = false;
  // Every lane stays in this loop until the whole warp is done, so the warp is
  // converged at the top of each iteration (one event per iteration).
  while (true) {
    __syncwarp();
    // ---- refill idle lanes (warp-aggregated)
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
        } else {
          ip = cand;
          if (A.isvacant[ip]) {
            have = false;  // vacant slot: nothing to do, take another next iteration
          } else {
            // ---- particle set-up, particle_advance.f90:141-202
            double x, y, z, mu, om, e, e0, wl;
            load_packet(A.prt + ip, x, y, z, mu, om, e, e0, wl);
            atomicAdd(&s_cnt[0], 1ull);
            int m = 0;
            long long poff = 0;
            if (MODELS) {  // models own consecutive slot ranges
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
            p.x = x; p.mu = mu; p.e = e; p.e0 = e0; p.wl = wl; p.dist = 0.0;
            p.ix = binsrch(x, X, vnx + 1, false);
            p.ig = binsrch(wl, A.wl, A.ng + 1, false);
            if (p.ix < 1 || p.ig < 1) {  // NaN position or wavelength: library code 1002
              if (A.errorfatal) atomicMin(&A.acc->ierr_key, ((unsigned long long)(ip + 1) << 32) | 1002u);
              A.isvacant[ip] = 1;
              p.ix = 1;
              p.ig = 1;
            }
            const bool bad = A.isvacant[ip] != 0;
            const double help = dxv(X, p.ix);
            const double tau = (A.sig[vco + p.ix - 1] + CAPd(A, p.ig, vco + p.ix)) * help;
            p.itype = (A.puretran || tau < A.tauddmc) ? 1 : 2;
            p.vx = (VX[p.ix - 1] * (X[p.ix] - x) + VX[p.ix] * (x - X[p.ix - 1])) / (X[p.ix] - X[p.ix - 1]);
            if (p.itype == 1) {
              const double labfact = 1.0 - p.vx * p.mu / pc_c;
              p.wl = p.wl * labfact;
              p.e = p.e / labfact;
              p.e0 = p.e0 / labfact;
            }
            p.stat = 0;
            p.idist = 0;
            istep = 0;
            nd_p = 0;
            nsw_p = 0;
            rng.init(A.seed + (unsigned long long)m * kModelSeedStride, (uint64_t)(ip - poff), sw);
            if (TRACE) h = 1469598103934665603ull;
            have = !bad;
          }
        }
      }
    }
    if (__all_sync(0xffffffffu, !have && queue_done)) break;
    if (!have) continue;
    // ---- one event, particle_advance.f90:204-268
    istep++;
    const MView v{vnx, vco, vxo};
    const int icold = vco + p.ix, igold = p.ig;  // cell over all models, 1-based
    double eraddens, jrad, eamp = 0.0;
    int ierr;
    if (p.itype == 1 || A.puretran) {
      transport11_dev(A, v, p, rng, eraddens, eamp, jrad, evelo, ierr);
      if (p.itype != 1) {
        nsw_p++;
        if (A.dogrdtally) atomicAdd(&A.methodswap[icold - 1], 1);
      }
      if (!A.noampfact && eamp != 0.0) atomicAdd(&A.eamp[icold - 1], eamp);
    } else {
      nd_p++;
      diffusion11_dev(A, v, p, rng, eraddens, jrad, evelo, ierr);
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
      if (t_ic > 0 && t_acc != 0.0) atomicAdd(&A.tally[t_ic - 1], t_acc);
      t_ic = icold;
      t_acc = 0.0;
    }
    t_acc = t_acc + eraddens;
    if (icold != j_ic || igold != j_ig) {
      if (j_ic > 0 && j_acc != 0.0) atomicAdd(&A.jrad[(size_t)(j_ic - 1) * A.ng + (j_ig - 1)], j_acc);
      j_ic = icold;
      j_ig = igold;
      j_acc = 0.0;
    }
    j_acc = j_acc + jrad;
    if (TRACE) {
      h = fnv_mix(h, p.idist);
      h = fnv_mix(h, p.itype);
      h = fnv_mix(h, p.ix);
      h = fnv_mix(h, p.ig);
      h = fnv_mix(h, p.stat);
    }
    if (p.itype == 1 && p.stat == 0) {
      if (p.x > A.xarr[vxo + p.ix] || p.x < A.xarr[vxo + p.ix - 1] || p.x != p.x) {
        if (ierr == 0) ierr = -99;
      }
    }
    if (ierr == -99) atomicAdd(&s_cnt[6], 1ull);
    if (ierr == 0 && A.max_steps > 0 && istep >= A.max_steps && p.stat == 0) ierr = 1001;
    if (ierr > 0) {
      if (A.errorfatal) {
        const unsigned long long key = ((unsigned long long)(ip + 1) << 32) | (unsigned)ierr;
        atomicMin(&A.acc->ierr_key, key);
      }
      p.stat = 2;
    }
    if (p.stat != 0) {
      // ---- particle end, particle_advance.f90:271-292
      atomicMax(&s_cnt[5], (unsigned long long)istep);
      atomicAdd(&s_cnt[2], (unsigned long long)(istep - nd_p));
      atomicAdd(&s_cnt[3], (unsigned long long)nd_p);
      if (nsw_p) atomicAdd(&s_cnt[4], (unsigned long long)nsw_p);
      if (TRACE) {
        A.trace_hash[ip] = h;
        A.trace_nstep[ip] = istep;
      }
      if (p.stat == 2) {
        A.isvacant[ip] = 1;
      } else {
        atomicAdd(&s_cnt[1], 1ull);
        atomicAdd(&s_sum[1], p.e);   // tot_eout
        atomicAdd(&s_sum[2], -p.e);  // tot_sflux
        store_flux_packet(A.prt + ip, p.mu, p.e, p.e0, p.wl);
      }
      have = false;
    }
  }
  // ---- flush
  if (t_ic > 0 && t_acc != 0.0) atomicAdd(&A.tally[t_ic - 1], t_acc);
  if (j_ic > 0 && j_acc != 0.0) atomicAdd(&A.jrad[(size_t)(j_ic - 1) * A.ng + (j_ig - 1)], j_acc);
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
}

// fluxtally.f:30-54; flux-grid histogram in shared memory, flushed once per block.
__global__ void fluxtally_kernel(long long npart, const slg_packet* __restrict__ prt,
                                 int32_t* __restrict__ isvacant, int flx_ng, const double* __restrict__ flx_wl,
                                 double* __restrict__ luminos, double* __restrict__ lumdev,
                                 int32_t* __restrict__ lumnum, int use_smem) {
  extern __shared__ double sh[];
  double* s_lum = sh;
  double* s_dev = sh + flx_ng;
  int* s_num = reinterpret_cast<int*>(sh + 2 * flx_ng);
  if (use_smem) {
    for (int k = threadIdx.x; k < flx_ng; k += blockDim.x) { s_lum[k] = 0.0; s_dev[k] = 0.0; s_num[k] = 0; }
    __syncthreads();
  }
  for (long long ip = (long long)blockIdx.x * blockDim.x + threadIdx.x; ip < npart;
       ip += (long long)gridDim.x * blockDim.x) {
    if (isvacant[ip]) continue;
    const slg_packet* q = prt + ip;
    if (q->x != DBL_MAX) continue;
    const double e = q->e;
    const int ig = binsrch(q->wl, flx_wl, flx_ng + 1, false);
    if (ig < 1) continue;  // NaN wavelength
    if (use_smem) {
      atomicAdd(&s_lum[ig - 1], e);
      atomicAdd(&s_dev[ig - 1], sq(e));
      atomicAdd(&s_num[ig - 1], 1);
    } else {
      atomicAdd(&luminos[ig - 1], e);
      atomicAdd(&lumdev[ig - 1], sq(e));
      atomicAdd(&lumnum[ig - 1], 1);
    }
    isvacant[ip] = 1;
  }
  if (use_smem) {
    __syncthreads();
    for (int k = threadIdx.x; k < flx_ng; k += blockDim.x) {
      if (s_num[k]) {
        atomicAdd(&luminos[k], s_lum[k]);
        atomicAdd(&lumdev[k], s_dev[k]);
        atomicAdd(&lumnum[k], s_num[k]);
      }
    }
  }
}

// sourcetally.f:24-45: src_energy/src_number (ncell, ng), cell fastest.
__global__ void sourcetally_kernel(long long npart, const slg_packet* __restrict__ prt,
                                   const int32_t* __restrict__ isvacant, int nx, int ng,
                                   const double* __restrict__ xarr, const double* __restrict__ wl,
                                   double* __restrict__ src_energy, int32_t* __restrict__ src_number,
                                   int* __restrict__ err, int nmodel, const ModelDesc* __restrict__ models) {
  for (long long ip = (long long)blockIdx.x * blockDim.x + threadIdx.x; ip < npart;
       ip += (long long)gridDim.x * blockDim.x) {
    if (isvacant[ip]) continue;
    const slg_packet* q = prt + ip;
    // the slot's model: shells mnx from cell co, edges from xo
    int mnx = nx, co = 0, xo = 0;
    if (nmodel > 1) {
      int lo = 0, hi = nmodel - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (models[mid].poff <= ip) lo = mid;
        else hi = mid - 1;
      }
      mnx = models[lo].nx;
      co = models[lo].co;
      xo = models[lo].xo;
    }
    const int ig = binsrch(q->wl, wl, ng + 1, false);
    const int ic = binsrch(q->x, xarr + xo, mnx + 1, false);
    if (ic < 1 || ic > mnx) { atomicOr(err, 1); continue; }
    if (ig < 1 || ig > ng) { atomicOr(err, 2); continue; }
    atomicAdd(&src_energy[(size_t)(ig - 1) * nx + (co + ic - 1)], q->e);
    atomicAdd(&src_number[(size_t)(ig - 1) * nx + (co + ic - 1)], 1);
  }
}

template <bool TRACE, int MINB, bool MODELS = false>
int launch_one(int num_sms, long long npart, cudaStream_t st, const TrnArgs& A) {
  static int occ = -1;  // resident blocks per SM, queried once (not during a capture)
  if (occ < 0)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, particle_advance_kernel<TRACE, MINB, MODELS>, TRN_BLOCK, 0);
  long long nblk = (long long)num_sms * (occ > 0 ? occ : 4);
  const long long need = (npart + TRN_BLOCK - 1) / TRN_BLOCK;
  if (need < nblk) nblk = need > 0 ? need : 1;
  particle_advance_kernel<TRACE, MINB, MODELS><<<(unsigned)nblk, TRN_BLOCK, 0, st>>>(A);
  return cudaPeekAtLastError() == cudaSuccess ? SLG_OK : SLG_ERR_CUDA;
}

}  // namespace

int launch_transport_mixed(int variant, int num_sms, long long npart, cudaStream_t st, const TrnArgs& A);
int launch_mix_rate_tables(cudaStream_t st, int nc, const int4* cellmap, const TrnArgs& A, float4* mrate,
                           float* emit32, int16_t* eguide);
constexpr int kMixedVariants = 4;

// Transport kernel variants (register budget / resident blocks), see MINB.
constexpr int kTransportVariants = 4;
int launch_transport_variant(int v, bool trace, int num_sms, long long npart, cudaStream_t st, const TrnArgs& A) {
  if (A.nmodel > 1) {  // several models: no per-event trace
    switch (v) {
      case 1: return launch_one<false, 5, true>(num_sms, npart, st, A);
      case 2: return launch_one<false, 6, true>(num_sms, npart, st, A);
      case 3: return launch_one<false, 8, true>(num_sms, npart, st, A);
      default: return launch_one<false, 1, true>(num_sms, npart, st, A);
    }
  }
  switch (v) {
    case 1: return trace ? launch_one<true, 5>(num_sms, npart, st, A) : launch_one<false, 5>(num_sms, npart, st, A);
    case 2: return trace ? launch_one<true, 6>(num_sms, npart, st, A) : launch_one<false, 6>(num_sms, npart, st, A);
    case 3: return trace ? launch_one<true, 8>(num_sms, npart, st, A) : launch_one<false, 8>(num_sms, npart, st, A);
    default: return trace ? launch_one<true, 1>(num_sms, npart, st, A) : launch_one<false, 1>(num_sms, npart, st, A);
  }
}

// Grids up to this many cells keep grd_tally in shared memory in the
// mixed-precision kernel (32 KiB per block).
constexpr int kSmemTallyCells = 4096;

// Kernel arguments of one particle_advance over the context's grid and models.
// MixCell records of every cell (over all models), after build_cell_tables.
__global__ void mix_cell_kernel(int nc, const int4* __restrict__ cellmap, const double* __restrict__ xarr,
                                const double* __restrict__ vxarr, const double* __restrict__ divv,
                                const double* __restrict__ sig, const double* __restrict__ tempinv,
                                const double* __restrict__ opaclump, const double* __restrict__ scal,
                                const int32_t* __restrict__ nlump, MixCell* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  int i = c + 1, nx = nc, co = 0, m = 0;
  if (cellmap) {
    const int4 cm = cellmap[c];
    i = cm.x;
    nx = cm.y;
    co = cm.z;
    m = cm.w;
  }
  const double* X = xarr + co + m;
  const double* VX = vxarr + co + m;
  const double* sc = scal + (size_t)SCAL_N * c;
  MixCell r;
  r.xa = X[i - 1];
  r.xb = X[i];
  r.vxa = VX[i - 1];
  r.vxb = VX[i];
  r.x0 = X[0];
  r.capgreyinv = sc[SCAL_CAPGREYINV];
  r.tinv = tempinv[c];
  r.nlump = nlump[c];
  r.pad = 0;
  r.dist = (float)(r.xb - r.xa);
  r.sig = (float)sig[c];
  r.emitlump = (float)sc[SCAL_EMITLUMP];
  r.caplump = (float)sc[SCAL_CAPLUMP];
  r.doplump = (float)sc[SCAL_DOPLUMP];
  r.o1 = (float)opaclump[(size_t)11 * c];
  r.o2 = (float)opaclump[(size_t)11 * c + 1];
  r.divv = (float)divv[c];
  r.far = (float)sc[SCAL_FAR];
  r.dvdr = (float)sc[SCAL_DVDR];
  r.sigl = i > 1 ? (float)sig[c - 1] : 0.f;
  r.sigr = i < nx ? (float)sig[c + 1] : 0.f;
  r.dxl = i > 1 ? (float)(r.xa - X[i - 2]) : 0.f;
  r.dxr = i < nx ? (float)(X[i + 1] - r.xb) : 0.f;
  r.fa = (float)(sq(r.xa) / sc[SCAL_DX3]);
  r.fb = (float)(sq(r.xb) / sc[SCAL_DX3]);
  out[c] = r;
}

// FP32 copies of the four running-sum tables (n entries each).
__global__ void cdf32_kernel(size_t n, const double* __restrict__ a0, const double* __restrict__ a1,
                             const double* __restrict__ a2, const double* __restrict__ a3, float* __restrict__ b0,
                             float* __restrict__ b1, float* __restrict__ b2, float* __restrict__ b3) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    b0[i] = (float)a0[i];
    b1[i] = (float)a1[i];
    b2[i] = (float)a2[i];
    b3[i] = (float)a3[i];
  }
}

// Builds the MixCell records and the FP32 running sums for a mixed-precision
// launch (scratch slots 76-80).
int build_mix_cells(slg_ctx* ctx, const slg_transport_in* in, TrnArgs& A) {
  const int nc = ctx->nx;
  auto* rec = (MixCell*)scratch(ctx, 76, sizeof(MixCell) * (size_t)nc);
  if (!rec) return SLG_ERR_OOM;
  const size_t n = (size_t)nc * ctx->ng;
  float* c32[4];
  for (int t = 0; t < 4; ++t) {
    c32[t] = (float*)scratch(ctx, 77 + t, sizeof(float) * n);
    if (!c32[t]) return SLG_ERR_OOM;
  }
  const CellTables& T = ctx->tables;
  long long nb = (long long)((n + 255) / 256);
  if (nb > 4LL * ctx->num_sms) nb = 4LL * ctx->num_sms;
  cdf32_kernel<<<(unsigned)(nb > 0 ? nb : 1), 256, 0, ctx->stream>>>(n, T.cdf_dop, T.cdf_left, T.cdf_right, T.cdf_scat,
                                                                    c32[0], c32[1], c32[2], c32[3]);
  A.T.cdf32_dop = c32[0];
  A.T.cdf32_left = c32[1];
  A.T.cdf32_right = c32[2];
  A.T.cdf32_scat = c32[3];
  mix_cell_kernel<<<(nc + 127) / 128, 128, 0, ctx->stream>>>(nc, ctx->nmodel > 1 ? ctx->d_cellmap : nullptr,
                                                            ctx->d_xarr, ctx->d_vxarr, ctx->d_divv, in->sig,
                                                            in->tempinv, in->opaclump, ctx->tables.scal,
                                                            ctx->tables.nlump, rec);
  A.mcell = rec;
  int rc = cuda_check(ctx, cudaGetLastError(), "mix_cell_kernel");
  if (rc) return rc;
  // per (cell, group) DDMC rates and per-cell emission CDFs (scratch slots 81-83)
  auto* mrate = (float4*)scratch(ctx, 81, sizeof(float4) * n);
  auto* emit32 = (float*)scratch(ctx, 82, sizeof(float) * n);
  auto* eguide = (int16_t*)scratch(ctx, 83, sizeof(int16_t) * (size_t)nc * (T.guide_m + 1));
  if (!mrate || !emit32 || !eguide) return SLG_ERR_OOM;
  A.mrate = mrate;
  A.emit32 = emit32;
  A.eguide = eguide;
  rc = launch_mix_rate_tables(ctx->stream, nc, ctx->nmodel > 1 ? ctx->d_cellmap : nullptr, A, mrate, emit32, eguide);
  return rc ? set_error(ctx, rc, "mixed rate tables: %s", cudaGetErrorString(cudaGetLastError())) : SLG_OK;
}

TrnArgs transport_args(slg_ctx* ctx, const slg_transport_in* in, slg_packet* prt, int32_t* isvacant,
                       long long npart, uint64_t seed, double* tally, double* jrad, double* eamp,
                       int32_t* methodswap) {
  TrnArgs A;
  A.nx = ctx->nx; A.ng = ctx->ng; A.nep = ctx->nep; A.nepg = ctx->nepg;
  A.xarr = ctx->d_xarr; A.vxarr = ctx->d_vxarr; A.divv = ctx->d_divv; A.wl = ctx->d_wl; A.wlinv = ctx->d_wlinv;
  A.tempinv = in->tempinv; A.sig = in->sig; A.capgrey = in->capgrey; A.emitprob = in->emitprob;
  A.opaclump = in->opaclump; A.cap = in->cap; A.tauddmc = in->tauddmc; A.taulump = in->taulump;
  A.puretran = in->puretran; A.noampfact = in->noampfact; A.errorfatal = in->errorfatal;
  A.thm_aniso = in->thm_aniso; A.dogrdtally = in->dogrdtally; A.max_steps = in->max_steps;
  A.T = ctx->tables; A.prt = prt; A.isvacant = isvacant; A.npart = npart; A.seed = seed;
  A.tally = tally; A.jrad = jrad; A.eamp = eamp; A.methodswap = methodswap;
  A.acc = ctx->d_acc; A.trace_hash = nullptr; A.trace_nstep = nullptr;
  A.epoch = ctx->capturing ? ctx->d_epoch : nullptr;
  A.nmodel = ctx->nmodel > 1 ? ctx->nmodel : 1;
  A.models = ctx->nmodel > 1 ? ctx->d_models : nullptr;
  A.smem_cells = ctx->nx <= kSmemTallyCells ? ctx->nx : 0;
  return A;
}

// Running sums of the transport counters over launches (sums, max of the
// longest history, first error).
__global__ void totals_fold_kernel(const TransportAcc* __restrict__ a, TransportAcc* __restrict__ t) {
  if (threadIdx.x == 0) {
    t->evelo += a->evelo; t->eout += a->eout; t->sflux += a->sflux;
    t->npckt += a->npckt; t->nflux += a->nflux; t->nimc += a->nimc; t->nddmc += a->nddmc;
    t->nswap += a->nswap; t->nwarn += a->nwarn;
    t->nmax = a->nmax > t->nmax ? a->nmax : t->nmax;
    if (a->ierr_key < t->ierr_key) t->ierr_key = a->ierr_key;  // all ones: no error
  }
  if (threadIdx.x < 11) t->ndist[threadIdx.x] += a->ndist[threadIdx.x];
}

int launch_particle_advance(slg_ctx* ctx, const slg_transport_in* in, slg_packet* prt, int32_t* isvacant,
                            int64_t npart, uint64_t seed, slg_transport_out* out, uint64_t* d_trace_hash,
                            int32_t* d_trace_nstep) {
  const int nx = ctx->nx, ng = ctx->ng;
  cudaStream_t st = ctx->stream;
  int rc = build_cell_tables(ctx, in);
  if (rc) return rc;
  cudaMemsetAsync(out->tally, 0, sizeof(double) * nx, st);
  cudaMemsetAsync(out->jrad, 0, sizeof(double) * (size_t)nx * ng, st);
  cudaMemsetAsync(out->eamp, 0, sizeof(double) * nx, st);
  if (in->dogrdtally && out->methodswap) cudaMemsetAsync(out->methodswap, 0, sizeof(int32_t) * nx, st);
  cudaMemsetAsync(ctx->d_acc, 0, sizeof(TransportAcc), st);
  cudaMemsetAsync(&ctx->d_acc->ierr_key, 0xff, sizeof(unsigned long long), st);
  TrnArgs A = transport_args(ctx, in, prt, isvacant, npart, seed, out->tally, out->jrad, out->eamp,
                             out->methodswap);
  A.trace_hash = d_trace_hash;
  A.trace_nstep = d_trace_nstep;
  if (in->precision == 1) {
    A.trace_hash = nullptr;  // the mixed form has no per-event trace
    A.trace_nstep = nullptr;
    if ((rc = build_mix_cells(ctx, in, A))) return rc;
    rc = launch_transport_mixed(ctx->mix_variant, ctx->num_sms, npart, st, A);
  } else {
    rc = launch_transport_variant(ctx->trn_variant, d_trace_hash != nullptr, ctx->num_sms, npart, st, A);
  }
  if (rc) return set_error(ctx, rc, "particle_advance launch: %s", cudaGetErrorString(cudaGetLastError()));
  totals_fold_kernel<<<1, 32, 0, st>>>(ctx->d_acc, ctx->d_totals);
  return cuda_check(ctx, cudaMemcpyAsync(ctx->h_acc, ctx->d_acc, sizeof(TransportAcc), cudaMemcpyDeviceToHost, st),
                    "transport counters download");
}

// After the stream has reached the end of launch_particle_advance: fold the
// device counters into *out (totals accumulate like totalsmod.f).
int finish_particle_advance(slg_ctx* ctx, const slg_transport_in* in, slg_transport_out* out) {
  (void)in;
  const TransportAcc& a = *ctx->h_acc;
  out->tot_evelo += a.evelo;
  out->tot_eout += a.eout;
  out->tot_sflux += a.sflux;
  out->npckt = (int64_t)a.npckt;
  out->nflux = (int64_t)a.nflux;
  out->nstepimc = (int64_t)a.nimc;
  out->nstepddmc = (int64_t)a.nddmc;
  out->nmethodswap = (int64_t)a.nswap;
  out->nstepmax = (int64_t)a.nmax;
  for (int k = 0; k < 11; ++k) out->ndist[k] = (int64_t)a.ndist[k];
  out->nposwarn = (int64_t)a.nwarn;
  if (a.ierr_key != ~0ull) {
    out->ierr = (int32_t)(a.ierr_key & 0xffffffffu);
    out->ierr_part = (int32_t)(a.ierr_key >> 32);
  } else {
    out->ierr = 0;
    out->ierr_part = 0;
  }
  return out->ierr;
}

int launch_fluxtally(slg_ctx* ctx, int64_t npart, const slg_packet* prt, int32_t* isvacant, int flx_ng,
                     const double* flx_wl, double* luminos, double* lumdev, int32_t* lumnum) {
  cudaStream_t st = ctx->stream;
  cudaMemsetAsync(luminos, 0, sizeof(double) * flx_ng, st);
  cudaMemsetAsync(lumdev, 0, sizeof(double) * flx_ng, st);
  cudaMemsetAsync(lumnum, 0, sizeof(int32_t) * flx_ng, st);
  const size_t shm = (size_t)flx_ng * (2 * sizeof(double) + sizeof(int));
  const int use_smem = shm <= 96 * 1024;
  static unsigned raised = 0;  // per device; no attribute calls on repeated launches
  if (use_smem) raise_smem_limit(raised, ctx->device, fluxtally_kernel, 96 * 1024);
  long long nb = (npart + 255) / 256;
  const long long cap = (long long)ctx->num_sms * 4;
  if (nb > cap) nb = cap;
  if (nb < 1) nb = 1;
  fluxtally_kernel<<<(unsigned)nb, 256, use_smem ? shm : 0, st>>>(npart, prt, isvacant, flx_ng, flx_wl, luminos,
                                                                  lumdev, lumnum, use_smem);
  return cuda_check(ctx, cudaGetLastError(), "fluxtally launch");
}

int launch_sourcetally(slg_ctx* ctx, int64_t npart, const slg_packet* prt, const int32_t* isvacant,
                       double* src_energy, int32_t* src_number) {
  cudaStream_t st = ctx->stream;
  const size_t n = (size_t)ctx->nx * ctx->ng;
  int* d_err = (int*)scratch(ctx, 21, sizeof(int) * 2);
  if (!d_err) return SLG_ERR_OOM;
  cudaMemsetAsync(d_err, 0, sizeof(int) * 2, st);
  cudaMemsetAsync(src_energy, 0, sizeof(double) * n, st);
  cudaMemsetAsync(src_number, 0, sizeof(int32_t) * n, st);
  long long nb = (npart + 255) / 256;
  const long long cap = (long long)ctx->num_sms * 8;
  if (nb > cap) nb = cap;
  if (nb < 1) nb = 1;
  if (ctx->nmodel > 1 && npart != ctx->npart_models)
    return set_error(ctx, SLG_ERR_ARG, "sourcetally: npart differs from the models' slots");
  sourcetally_kernel<<<(unsigned)nb, 256, 0, st>>>(npart, prt, isvacant, ctx->nx, ctx->ng, ctx->d_xarr, ctx->d_wl,
                                                   src_energy, src_number, d_err,
                                                   ctx->nmodel > 1 ? ctx->nmodel : 1, ctx->d_models);
  return cuda_check(ctx, cudaGetLastError(), "sourcetally launch");
}

int sourcetally_error(slg_ctx* ctx, int* err) {
  int* d_err = (int*)scratch(ctx, 21, sizeof(int) * 2);
  int h = 0;
  int rc = cuda_check(ctx, cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "err");
  if (rc) return rc;
  rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  *err = h;
  return rc;
}

}  // namespace slg

namespace slg {
// Launch of particle_advance_kernel with every buffer supplied by the caller
// (used by the entry point that allocates nothing).  nblk is the grid size.
int launch_particle_advance_raw(cudaStream_t st, const TrnArgs& A, int nblk) {
  particle_advance_kernel<false, 1><<<(unsigned)nblk, TRN_BLOCK, 0, st>>>(A);
  return cudaGetLastError() == cudaSuccess ? SLG_OK : SLG_ERR_CUDA;
}
int particle_advance_blocks_per_sm() {
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, particle_advance_kernel<false, 1>, TRN_BLOCK, 0);
  return occ > 0 ? occ : 4;
}
int particle_advance_block_size() { return TRN_BLOCK; }

// Autotuner of the transport kernel: runs every variant of
// launch_transport_variant on the same copy of (a sample of) the caller's
// particles, times each with CUDA events and keeps the fastest for this
// context.  Device pointers; results are discarded.
int autotune_transport(slg_ctx* ctx, const slg_transport_in* in, const slg_packet* prt, const int32_t* isvacant,
                       int64_t npart, uint64_t seed, int64_t nsample, int* best, float* ms) {
  const int nx = ctx->nx, ng = ctx->ng;
  cudaStream_t st = ctx->stream;
  int rc = build_cell_tables(ctx, in);
  if (rc) return rc;
  const long long n = nsample > 0 && nsample < npart ? nsample : npart;
  slg_packet* p = (slg_packet*)scratch(ctx, 40, sizeof(slg_packet) * (n > 0 ? n : 1));
  int32_t* v = (int32_t*)scratch(ctx, 41, sizeof(int32_t) * (n > 0 ? n : 1));
  double* tally = (double*)scratch(ctx, 42, sizeof(double) * nx);
  double* jrad = (double*)scratch(ctx, 43, sizeof(double) * (size_t)nx * ng);
  double* eamp = (double*)scratch(ctx, 44, sizeof(double) * nx);
  int32_t* msw = (int32_t*)scratch(ctx, 45, sizeof(int32_t) * nx);
  if (!p || !v || !tally || !jrad || !eamp || !msw) return SLG_ERR_OOM;
  TrnArgs A = transport_args(ctx, in, p, v, n, seed, tally, jrad, eamp, msw);
  const bool mixed = in->precision == 1;
  if (mixed && (rc = build_mix_cells(ctx, in, A))) return rc;
  const int nvar = mixed ? kMixedVariants : kTransportVariants;
  cudaEvent_t e0, e1;
  if ((rc = cuda_check(ctx, cudaEventCreate(&e0), "event"))) return rc;
  if ((rc = cuda_check(ctx, cudaEventCreate(&e1), "event"))) { cudaEventDestroy(e0); return rc; }
  float bestms = 0.f;
  int bestv = 0;
  for (int var = 0; var < nvar && !rc; ++var) {
    cudaMemcpyAsync(p, prt, sizeof(slg_packet) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(v, isvacant, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemsetAsync(tally, 0, sizeof(double) * nx, st);
    cudaMemsetAsync(jrad, 0, sizeof(double) * (size_t)nx * ng, st);
    cudaMemsetAsync(ctx->d_acc, 0, sizeof(TransportAcc), st);
    cudaEventRecord(e0, st);
    rc = mixed ? launch_transport_mixed(var, ctx->num_sms, n, st, A)
               : launch_transport_variant(var, false, ctx->num_sms, n, st, A);
    cudaEventRecord(e1, st);
    if (!rc) rc = cuda_check(ctx, cudaEventSynchronize(e1), "autotune sync");
    float t = 0.f;
    if (!rc) cudaEventElapsedTime(&t, e0, e1);
    if (ms) ms[var] = t;
    if (!rc && (var == 0 || t < bestms)) { bestms = t; bestv = var; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (mixed) ctx->mix_variant = bestv;
  else ctx->trn_variant = bestv;
  if (best) *best = bestv;
  return SLG_OK;
}

// Fold device counters read back by the caller into *out (totals accumulate).
int finish_particle_advance_acc(const TransportAcc& a, slg_transport_out* out) {
  out->tot_evelo += a.evelo;
  out->tot_eout += a.eout;
  out->tot_sflux += a.sflux;
  out->npckt = (int64_t)a.npckt;
  out->nflux = (int64_t)a.nflux;
  out->nstepimc = (int64_t)a.nimc;
  out->nstepddmc = (int64_t)a.nddmc;
  out->nmethodswap = (int64_t)a.nswap;
  out->nstepmax = (int64_t)a.nmax;
  for (int k = 0; k < 11; ++k) out->ndist[k] = (int64_t)a.ndist[k];
  out->nposwarn = (int64_t)a.nwarn;
  out->ierr = a.ierr_key != ~0ull ? (int32_t)(a.ierr_key & 0xffffffffu) : 0;
  out->ierr_part = a.ierr_key != ~0ull ? (int32_t)(a.ierr_key >> 32) : 0;
  return out->ierr;
}
}  // namespace slg
