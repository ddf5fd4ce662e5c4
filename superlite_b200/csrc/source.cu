// source.cu -- source-particle creation on the GPU: sourceenergy,
// sourcenumbers (host, O(ncell)), vacancies, interior_source and
// source_transformdirection, for sm_100a.
//
// Reference: SOURCE/sourceenergy.f90:21-29, SOURCE/sourcenumbers.f90:3-94
// (one rank, no surface source), SOURCE/vacancies.f90:3-30,
// SOURCE/interior_source.f90:3-172, SOURCE/source_transformdirection.f90:3-47,
// transportmod.f:129-145 (direction2lab1).
//
// The reference draws every source particle from one sequential mzran stream
// on the host.  Here particle k (k-th new particle, filling the k-th vacant
// slot ivac) draws from its own Philox stream (seed, pid = ivac-1, stream 1)
// in the reference's draw order, so any number of particles are made in
// parallel and the CPU oracle reproduces them exactly.
#include <cuda_runtime.h>
#include <algorithm>
#include <cfloat>
#include <cmath>
#include "slg_device.cuh"
#include "slg_internal.h"

namespace slg {
namespace {

constexpr int SB = 256;

// per-cell normalised Planck weights, then their running sum in the order of
// interior_source.f90:177-181,202-209 (one block per emitting cell)
__global__ void __launch_bounds__(SB) source_cdf_kernel(int nx, int ng, const double* __restrict__ radtemp,
                                                        const double* __restrict__ wlinv,
                                                        const int32_t* __restrict__ nvol,
                                                        double* __restrict__ cdf) {
  const int l = blockIdx.x;
  if (nvol[l] < 1) return;
  double* c = cdf + (size_t)l * ng;
  const double tradinv = 1.0 / radtemp[l];
  const double hct = hck * tradinv;
  for (int g = threadIdx.x; g < ng; g += SB) c[g] = specintv_elem(hct, wlinv, g);
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int g = 0; g < ng; ++g) s = s + c[g];
    double denom2 = 0.0;
    for (int g = 0; g < ng; ++g) {
      denom2 = denom2 + c[g] / s;
      c[g] = denom2;
    }
  }
}

// vacancies.f90: the first nnew vacant slots in index order.
// Pass 1: vacant count per block of 1024 slots.
__global__ void vacancy_count_kernel(long long npart, const int32_t* __restrict__ isvacant,
                                     unsigned int* __restrict__ counts) {
  __shared__ unsigned int s;
  if (threadIdx.x == 0) s = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * 1024;
  unsigned int n = 0;
  for (int k = threadIdx.x; k < 1024; k += blockDim.x) {
    const long long ip = base + k;
    if (ip < npart && isvacant[ip]) ++n;
  }
  atomicAdd(&s, n);
  __syncthreads();
  if (threadIdx.x == 0) counts[blockIdx.x] = s;
}

// Pass 2: exclusive scan of the block counts (one block, sequential chunks).
__global__ void __launch_bounds__(1024) vacancy_scan_kernel(int nblk, unsigned int* __restrict__ counts,
                                                            unsigned long long* __restrict__ total) {
  __shared__ unsigned long long part[1024];
  const int per = (nblk + 1023) / 1024;
  const int b = threadIdx.x * per;
  unsigned long long s = 0;
  for (int k = b; k < b + per && k < nblk; ++k) s += counts[k];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long acc = 0;
    for (int t = 0; t < 1024; ++t) {
      const unsigned long long v = part[t];
      part[t] = acc;
      acc += v;
    }
    *total = acc;
  }
  __syncthreads();
  unsigned long long acc = part[threadIdx.x];
  for (int k = b; k < b + per && k < nblk; ++k) {
    const unsigned int v = counts[k];
    counts[k] = (unsigned int)acc;  // offsets fit in 32 bits per 2^32 particles
    acc += v;
  }
}

// Pass 3: write the ordered vacancy list (one warp per 1024-slot block keeps order).
__global__ void vacancy_write_kernel(long long npart, const int32_t* __restrict__ isvacant,
                                     const unsigned int* __restrict__ offsets, long long nnew,
                                     long long* __restrict__ ivacant) {
  const int lane = threadIdx.x & 31;
  const long long base = (long long)blockIdx.x * 1024;
  long long pos = offsets[blockIdx.x];
  if (threadIdx.x >= 32) return;
  for (int c = 0; c < 1024; c += 32) {
    const long long ip = base + c + lane;
    const bool v = ip < npart && isvacant[ip];
    const unsigned m = __ballot_sync(0xffffffffu, v);
    if (v) {
      const long long q = pos + __popc(m & ((1u << lane) - 1u));
      if (q < nnew) ivacant[q] = ip;
    }
    pos += __popc(m);
  }
}

struct SrcArgs {
  int nx, ng;
  const double *xarr, *vxarr, *wlinv, *emit, *cdf;
  const int32_t* nvol;
  const long long* cstart;  // first new-particle index of each cell (nx+1)
  const long long* ivacant;
  long long nnew;
  uint64_t seed;
  slg_packet* prt;
  int32_t* isvacant;
  int* flags;
  // several models: per-cell map {shell, model shells, model first cell,
  // model}, model descriptors and the count of vacant slots before each
  // model's first slot; null for one model
  const int4* cellmap;
  const ModelDesc* models;
  const unsigned long long* vbase;
  const unsigned long long* epoch;  // replay counter of a captured graph (may be null)
};

// Vacant slots before each model's first slot (vbase[nmodel] = all), from the
// scanned 1024-slot block counts and a count inside the block.
__global__ void model_vacancy_base_kernel(int nmodel, long long npart, const int32_t* __restrict__ isvacant,
                                          const ModelDesc* __restrict__ models, int nblk,
                                          const unsigned int* __restrict__ offsets,
                                          const unsigned long long* __restrict__ total,
                                          unsigned long long* __restrict__ vbase) {
  const int m = blockIdx.x;
  const long long p0 = m < nmodel ? models[m].poff : npart;
  const long long b = p0 / 1024;
  if (b >= nblk) {
    if (threadIdx.x == 0) vbase[m] = *total;
    return;
  }
  unsigned int n = 0;
  for (long long ip = b * 1024 + threadIdx.x; ip < p0; ip += 32) n += isvacant[ip] != 0;
  for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
  if (threadIdx.x == 0) vbase[m] = offsets[b] + n;
}

// interior_source.f90:193-268 and source_transformdirection.f90:20-44
__global__ void __launch_bounds__(SB) source_particle_kernel(const SrcArgs A) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= A.nnew) return;
  // cell i (1-based) with cstart[i-1] <= k < cstart[i]
  int lo = 0, hi = A.nx;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (A.cstart[mid] <= k) lo = mid;
    else hi = mid;
  }
  int i = lo + 1;  // shell within the model from here on
  int nx = A.nx, co = 0, m = 0;
  long long poff = 0, kv = k;  // kv: rank of the slot among the model's vacancies
  const double *xarr = A.xarr, *vxarr = A.vxarr, *emit = A.emit;
  const int32_t* nvol = A.nvol;
  if (A.cellmap) {
    const int4 cm = A.cellmap[lo];
    co = cm.z;
    m = cm.w;
    i = cm.x;
    nx = cm.y;
    poff = A.models[m].poff;
    kv = (long long)A.vbase[m] + (k - A.cstart[co]);
    if (kv >= (long long)A.vbase[m + 1]) {  // fewer vacancies than new particles in the model
      atomicOr(A.flags, 2);
      return;
    }
    xarr += co + m;
    vxarr += co + m;
    emit += co;
    nvol += co;
  }
  const long long ivac = A.ivacant[kv];
  PhiloxStream rng;
  rng.init(A.seed + (unsigned long long)m * kModelSeedStride, (uint64_t)(ivac - poff),
           1u | (A.epoch ? (uint32_t)(*A.epoch << 2) : 0u));
  const double* c = A.cdf + (size_t)(co + i - 1) * A.ng;
  double r1 = rng.draw();
  int a = 0, b = A.ng;  // first g with c[g] > r1, else the last group
  while (a < b) {
    const int mid = (a + b) >> 1;
    if (c[mid] > r1) b = mid;
    else a = mid + 1;
  }
  const int iig = a < A.ng ? a + 1 : A.ng;
  r1 = rng.draw();
  const double wl0 = 1.0 / ((1.0 - r1) * A.wlinv[iig - 1] + r1 * A.wlinv[iig]);
  const int nemit = nvol[i - 1];
  const double ep0 = emit[i - 1] / (double)nemit;
  r1 = rng.draw();
  const double mu0 = sqrt(r1);
  r1 = rng.draw();
  const double om0 = pc_pi2 * r1;
  const int icnb1 = max(i - 1, 1), icnb2 = min(i + 1, nx);
  const double el = emit[i - 1];
  double uul = 0.5 * (emit[icnb1 - 1] + el);
  double uur = 0.5 * (emit[icnb2 - 1] + el);
  const double uumax = uul > uur ? uul : uur;
  uul = uul / uumax;
  uur = uur / uumax;
  const double Xa = xarr[i - 1], Xb = xarr[i];
  double r3 = 0.0, r2 = 1.0, x0 = Xa;
  int guard = 0;
  while (r2 > r3) {
    r1 = rng.draw();
    x0 = pow(r1 * cube(Xb) + (1.0 - r1) * cube(Xa), third_r4);
    r3 = (x0 - Xa) / (Xb - Xa);
    r3 = r3 * uur + (1.0 - r3) * uul;
    r2 = rng.draw();
    if (++guard > 100000) { atomicOr(A.flags, 1); break; }  // acceptance is >= 1/4 in practice
  }
  // direction2lab1 on the interpolated velocity (source_transformdirection.f90:309-324)
  const int ix = binsrch(x0, xarr, nx + 1, false);
  const double vx = (vxarr[ix - 1] * (xarr[ix] - x0) + vxarr[ix] * (x0 - xarr[ix - 1])) /
                    (xarr[ix] - xarr[ix - 1]);
  const double cmffact = 1.0 + mu0 * vx * cinv;
  double mu = (mu0 + vx * cinv) / cmffact;
  mu = mu < 1.0 ? mu : 1.0;
  mu = mu > -1.0 ? mu : -1.0;
  double2* q = reinterpret_cast<double2*>(A.prt + ivac);
  q[0] = make_double2(x0, -1.0);  // y = grd_yarr(1) of a 1-D grid
  q[1] = make_double2(0.0, mu);   // z = grd_zarr(1)
  q[2] = make_double2(om0, ep0);
  q[3] = make_double2(ep0, wl0);
  A.isvacant[ivac] = 0;
}

}  // namespace

// sourceenergy.f90:21-29 on the host (O(ncell)).
void host_sourceenergy(int nx, const double* xarr, const double* radtemp, double L_bol, double* emit,
                       double* tot_sthermal) {
  double s = 0.0;
  for (int i = 0; i < nx; ++i) {
    const double rcell = (xarr[i + 1] + xarr[i]) / 2.0;
    emit[i] = pc_pi * pc_c * sq(rcell) * pc_acoef * pow4(radtemp[i]);
  }
  for (int i = 0; i < nx; ++i) s = s + emit[i];
  for (int i = 0; i < nx; ++i) emit[i] = emit[i] / s * L_bol;
  double t = 0.0;
  for (int i = 0; i < nx; ++i) t = t + emit[i];
  if (tot_sthermal) *tot_sthermal = t;
}

// sourcenumbers.f90:3-94 for a single rank without a surface source.
long long host_sourcenumbers(int nx, const double* emit, double pwr, long long src_ns, long long nvacant,
                             int32_t* nvol) {
  for (int l = 0; l < nx; ++l) nvol[l] = 0;
  double etot = 0.0;
  for (int l = 0; l < nx; ++l) etot = etot + std::pow(emit[l], pwr);
  etot = etot + std::pow(0.0, pwr);
  long long ncactive = 0;
  for (int l = 0; l < nx; ++l) ncactive += emit[l] > 0.0;
  if (ncactive == 0 || nvacant < ncactive) return -1;
  const long long nsavail = src_ns;
  double edone = 0.0;
  long long ndone = 0;
  const double invn = 1.0 / (double)nsavail;
  double einv = 1.0 / etot;
  if (etot == 0.0) einv = 0.0;
  for (int l = 0; l < nx; ++l) {
    const double en = std::pow(emit[l], pwr);
    if (en == 0.0) continue;
    long long n = (long long)(en * (double)nsavail * einv);
    if (n < 1) n = 1;
    if (edone * einv > (double)ndone * invn) n = n + 1;
    nvol[l] = (int32_t)n;
    edone = edone + en;
    ndone = ndone + n;
  }
  if (ndone == 0) return -2;
  long long sum = 0;
  for (int l = 0; l < nx; ++l) sum += nvol[l];
  long long nextra = src_ns - sum;
  if (nextra > nx) return -3;
  const long long nsmean = src_ns / ncactive;
  int guard = 0;
  while (nextra != 0) {
    for (int l = 0; l < nx; ++l) {
      if (nextra == 0) break;
      if (nvol[l] < nsmean) continue;
      const int s = nextra > 0 ? 1 : -1;
      nvol[l] += s;
      nextra -= s;
    }
    if (++guard > 1000000) return -4;
  }
  long long nnew = 0;
  for (int l = 0; l < nx; ++l)
    if (emit[l] != 0.0) nnew += nvol[l];
  return nnew;
}

int launch_interior_source(slg_ctx* ctx, const double* d_radtemp, const double* h_emit, const int32_t* h_nvol,
                           long long npart, slg_packet* prt, int32_t* isvacant, uint64_t seed, long long* nnew_out) {
  const int nx = ctx->nx, ng = ctx->ng;
  const bool models = ctx->nmodel > 1;
  cudaStream_t st = ctx->stream;
  std::vector<long long> cstart(nx + 1, 0);
  for (int l = 0; l < nx; ++l) {
    const long long n = h_emit[l] != 0.0 ? h_nvol[l] : 0;
    cstart[l + 1] = cstart[l] + n;
  }
  const long long nnew = cstart[nx];
  if (nnew > npart) return set_error(ctx, SLG_ERR_ARG, "interior_source: %lld new particles > %lld slots", nnew, npart);
  if (models) {
    if (npart != ctx->npart_models)
      return set_error(ctx, SLG_ERR_ARG, "interior_source: npart differs from the models' slots");
    for (int m = 0; m < ctx->nmodel; ++m) {
      const ModelDesc& d = ctx->h_models[m];
      const long long nm = cstart[d.co + d.nx] - cstart[d.co];
      if (nm > d.np)
        return set_error(ctx, SLG_ERR_ARG, "interior_source: model %d: %lld new particles > %lld slots", m, nm, d.np);
    }
  }
  *nnew_out = nnew;
  std::vector<int32_t> nv(nx);
  for (int l = 0; l < nx; ++l) nv[l] = h_emit[l] != 0.0 ? h_nvol[l] : 0;
  // all vacancies are listed for several models (each model takes its own)
  const long long nlist = models ? npart : nnew;
  double* d_emit = (double*)scratch(ctx, 22, sizeof(double) * nx);
  int32_t* d_nvol = (int32_t*)scratch(ctx, 23, sizeof(int32_t) * nx);
  long long* d_cstart = (long long*)scratch(ctx, 24, sizeof(long long) * (nx + 1));
  double* d_cdf = (double*)scratch(ctx, 25, sizeof(double) * (size_t)nx * ng);
  const long long nblk = (npart + 1023) / 1024;
  unsigned int* d_cnt = (unsigned int*)scratch(ctx, 26, sizeof(unsigned int) * (nblk > 0 ? nblk : 1));
  unsigned long long* d_tot = (unsigned long long*)scratch(ctx, 27, 64);
  long long* d_ivac = (long long*)scratch(ctx, 28, sizeof(long long) * (nlist > 0 ? nlist : 1));
  unsigned long long* d_vbase =
      models ? (unsigned long long*)scratch(ctx, 29, sizeof(unsigned long long) * (ctx->nmodel + 1)) : nullptr;
  int* d_flags = (int*)(d_tot + 2);
  if (!d_emit || !d_nvol || !d_cstart || !d_cdf || !d_cnt || !d_tot || !d_ivac || (models && !d_vbase))
    return SLG_ERR_OOM;
  if (nnew == 0) return SLG_OK;
  if (nblk > 0x7fffffffLL) return set_error(ctx, SLG_ERR_ARG, "too many particle slots");
  // the set-up is uploaded only when it changed, so repeated (and captured)
  // steps hold no host-to-device copies
  const bool same = ctx->src_emit.size() == (size_t)nx && ctx->src_nvol.size() == (size_t)nx &&
                    std::equal(nv.begin(), nv.end(), ctx->src_nvol.begin()) &&
                    std::equal(h_emit, h_emit + nx, ctx->src_emit.begin());
  if (!same) {
    if (ctx->capturing)
      return set_error(ctx, SLG_ERR_STATE, "interior_source: the source set-up changed during a graph capture");
    ctx->src_emit.clear();
    ctx->src_nvol.clear();
    int rc = cuda_check(ctx, cudaMemcpyAsync(d_emit, h_emit, sizeof(double) * nx, cudaMemcpyHostToDevice, st), "emit");
    if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(d_nvol, nv.data(), sizeof(int32_t) * nx, cudaMemcpyHostToDevice, st), "nvol");
    if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(d_cstart, cstart.data(), sizeof(long long) * (nx + 1),
                                                  cudaMemcpyHostToDevice, st), "cstart");
    // (copies from pageable memory return once the host data is staged)
    if (rc) return rc;
    ctx->src_emit.assign(h_emit, h_emit + nx);
    ctx->src_nvol = nv;
  }
  cudaMemsetAsync(d_tot, 0, 64, st);
  source_cdf_kernel<<<nx, SB, 0, st>>>(nx, ng, d_radtemp, ctx->d_wlinv, d_nvol, d_cdf);
  vacancy_count_kernel<<<(unsigned)nblk, 256, 0, st>>>(npart, isvacant, d_cnt);
  vacancy_scan_kernel<<<1, 1024, 0, st>>>((int)nblk, d_cnt, d_tot);
  vacancy_write_kernel<<<(unsigned)nblk, 32, 0, st>>>(npart, isvacant, d_cnt, nlist, d_ivac);
  if (models)
    model_vacancy_base_kernel<<<ctx->nmodel + 1, 32, 0, st>>>(ctx->nmodel, npart, isvacant, ctx->d_models,
                                                             (int)nblk, d_cnt, d_tot, d_vbase);
  SrcArgs A{nx, ng, ctx->d_xarr, ctx->d_vxarr, ctx->d_wlinv, d_emit, d_cdf, d_nvol, d_cstart, d_ivac, nnew, seed,
            prt, isvacant, d_flags, models ? ctx->d_cellmap : nullptr, models ? ctx->d_models : nullptr, d_vbase,
            ctx->capturing ? ctx->d_epoch : nullptr};
  source_particle_kernel<<<(unsigned)((nnew + SB - 1) / SB), SB, 0, st>>>(A);
  return cuda_check(ctx, cudaGetLastError(), "interior_source launch");
}

int interior_source_check(slg_ctx* ctx, long long nnew) {
  unsigned long long h[3] = {0, 0, 0};
  unsigned long long* d_tot = (unsigned long long*)scratch(ctx, 27, 64);
  int rc = cuda_check(ctx, cudaMemcpyAsync(h, d_tot, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream), "vac total");
  if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
  if (rc) return rc;
  if ((long long)h[0] < nnew) return set_error(ctx, SLG_ERR_ARG, "vacancies: %llu vacant slots < %lld new particles", h[0], nnew);
  if ((int)h[2] & 1) return set_error(ctx, SLG_ERR_CUDA, "interior_source: position rejection did not converge");
  if ((int)h[2] & 2) return set_error(ctx, SLG_ERR_ARG, "interior_source: a model has fewer vacant slots than new particles");
  return SLG_OK;
}

}  // namespace slg
