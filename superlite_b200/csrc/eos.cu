// eos.cu -- LTE equation of state (Saha ionisation balance) for sm_100a.
//
// Reference: ionsmod.f:160-356 (ions_solve_eos and its contained saha_nelec)
// and GAS/eos_update.f:20-45 (ground-state occupation densities).
//
// One warp per cell; lane iz-1 carries element iz's chain of stage
// populations, so the per-element recursions run side by side.  The electron
// count nelec = sum_iz natomfr(iz) ne(iz) is summed in element order (one
// shuffle per element) and every lane runs the same secant/overshoot update
// of the reference on the same values, so the warp stays converged.
//
// The partition functions are an input: the reference evaluates them only
// while they are all zero (ionsmod.f:209), i.e. once, at the temperature of
// the first cell of its first call, and reuses them afterwards.
// slg_partition_functions evaluates them at a given temperature.
#include <cuda_runtime.h>
#include <cfloat>
#include <cmath>
#include <vector>
#include "slg_device.cuh"
#include "slg_internal.h"

namespace slg {
namespace {

constexpr int EOS_MAXST = 32;  // stage slots per element (Z <= 30 has at most 31 stages)
constexpr int EOS_BLOCK = 128;

struct EosArgs {
  int nc, nelem, nstage, noc;
  const int32_t* ni;
  const double *e, *q, *g1;                    // (nstage, nelem)
  const double *temp, *natom, *vol, *natomfr;  // natomfr (0:nelem, ncell)
  double acc;
  double* nelec;  // in/out
  double* oc;     // (ncell, noc, nelem)
  double* ginv;
  int32_t* iconv;  // optional
  int* flags;      // bit 1: a cell where the reference stops (invalid sum, nelec <= 0)
};

__global__ void __launch_bounds__(EOS_BLOCK) saha_eos_kernel(const EosArgs A) {
  const int lane = threadIdx.x & 31;
  const int i = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (i >= A.nc) return;  // uniform over the warp
  const bool act = lane < A.nelem;
  const int ns = A.nstage;
  const int nion = act ? A.ni[lane] : 0;
  const double* e = A.e + (size_t)lane * ns;
  const double* q = A.q + (size_t)lane * ns;
  const double fr = act ? A.natomfr[(size_t)i * (A.nelem + 1) + lane + 1] : 0.0;
  const double T = A.temp[i];
  const double ndens = A.natom[i] / A.vol[i];
  const double kti = 1.0 / (pc_kb * T);
  const double sahac = pow(pc_pi2 * pc_me * pc_kb * T / (pc_h * pc_h), 1.5);
  double n[EOS_MAXST];
  double nel = A.nelec[i];
  double nec_nel0 = 0.0, nec_nel1 = 0.0, nec_err0 = 1e10, nec_err1 = -1e10;
  int iprev = 0, iconv, bad = 0;
  for (iconv = 1; iconv <= 40; ++iconv) {
    const double sahac2 = 2.0 / (nel * ndens) * sahac;
    // saha_nelec (ionsmod.f:298-354) for this lane's element
    double ne = 0.0;
    int inval = 0;
    if (act) {
      double help = 0.0;
      for (int istart = 1; istart <= nion - 1; ++istart) {
        n[istart - 1] = 1.0;
        for (int ii = istart + 1; ii <= nion; ++ii) {
          help = sahac2 * exp(-kti * e[ii - 2]) * n[ii - 2] * q[ii - 1] / q[ii - 2];
          n[ii - 1] = help;
        }
        if (help < DBL_MAX) break;
      }
      double nsum = 0.0;
      for (int ii = 0; ii < nion; ++ii) nsum = nsum + n[ii];
      if (nsum != nsum || nsum > DBL_MAX || nsum < DBL_MIN) inval = 1;
      nsum = 1.0 / nsum;
      for (int ii = 0; ii < nion; ++ii) n[ii] = n[ii] * nsum;
      for (int ii = 2; ii <= nion; ++ii) ne = ne + (double)(ii - 1) * n[ii - 1];
    }
    if (__any_sync(0xffffffffu, inval)) { bad = 1; break; }
    const double term = fr * ne;
    double nel_new = 0.0;
    for (int z = 0; z < A.nelem; ++z) nel_new = nel_new + __shfl_sync(0xffffffffu, term, z);
    const double err = nel / nel_new - 1.0;
    if (fabs(err) < A.acc) {
      if (iconv > 1) nel = nel_new;
      break;
    }
    // keep the bracket value on the same side of zero (maxloc(err*nec%err))
    if (err * nec_err1 > err * nec_err0) { nec_nel1 = nel; nec_err1 = err; }
    else { nec_nel0 = nel; nec_err0 = err; }
    if (iconv == 1) {
      nel = 1.5 * nel_new - 0.5 * nel;  // overshoot to bracket the root
      nel = fmin(3.0 * nel_new, nel);
      nel = fmax(0.33 * nel_new, nel);
    } else {
      const int ib = fabs(nec_err1) > fabs(nec_err0) ? 2 : 1;
      const double help = fabs(nec_err0 / nec_err1);
      const double ynew = (ib != iprev && help < 1e5 && help > 1e-5) ? 0.0 : 0.001 * (ib == 2 ? nec_err1 : nec_err0);
      iprev = ib;
      const double dxdy = (nec_nel1 - nec_nel0) / (nec_err1 - nec_err0);
      nel = nec_nel0 - dxdy * (nec_err0 - ynew);
      if (nel <= 0.0) { bad = 1; break; }
    }
  }
  if (bad) {
    if (lane == 0) {
      atomicOr(A.flags, 1);
      if (A.iconv) A.iconv[i] = -1;
    }
    return;
  }
  if (lane == 0) {
    A.nelec[i] = nel;
    if (A.iconv) A.iconv[i] = iconv;
  }
  if (!act) return;
  // eos_update.f:37-45, stages 1..noc of this element
  const double* g1 = A.g1 + (size_t)lane * ns;
  const double na = A.natom[i], v = A.vol[i];
  for (int ii = 0; ii < A.noc; ++ii) {
    const size_t o = (size_t)i + (size_t)A.nc * ((size_t)ii + (size_t)A.noc * lane);
    if (ii < nion) {
      A.ginv[o] = 1.0 / g1[ii];
      A.oc[o] = na * fr * g1[ii] * n[ii] / (q[ii] * v);
    } else {
      A.ginv[o] = 1.0;
      A.oc[o] = 0.0;
    }
  }
}

// Adjoint of the converged ionisation balance (no reference counterpart).
// With s = 2 sahac(T) / (nelec ndens) and c_k = exp(-e_k/kT) q_(k+1)/q_k, the
// stage fractions are f_k ~ s^(k-1) prod_(j<k) c_j (partition functions are
// constants, as in the reference), and nelec solves nelec = sum_z fr_z ne_z.
// Inputs: goc (ncell, noc, nelem) and gnelec (ncell) = dL/d(oc, nelec);
// outputs (added to): gT, gnatom (through ndens = natom/vol and oc), gfr
// (0:nelem, ncell).  One warp per cell, lane = element.
__global__ void __launch_bounds__(EOS_BLOCK) saha_eos_bwd_kernel(const EosArgs A, const double* __restrict__ goc,
                                                                const double* __restrict__ gnelec,
                                                                double* __restrict__ gT,
                                                                double* __restrict__ gnatom,
                                                                double* __restrict__ gfr) {
  const int lane = threadIdx.x & 31;
  const int i = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (i >= A.nc) return;
  const bool act = lane < A.nelem;
  const int ns = A.nstage;
  const int nion = act ? A.ni[lane] : 0;
  const double* e = A.e + (size_t)lane * ns;
  const double* q = A.q + (size_t)lane * ns;
  const double* g1 = A.g1 + (size_t)lane * ns;
  const double fr = act ? A.natomfr[(size_t)i * (A.nelem + 1) + lane + 1] : 0.0;
  const double T = A.temp[i], vol = A.vol[i];
  const double D = A.natom[i] / vol;
  const double kt = pc_kb * T;
  const double y = A.nelec[i];
  const double sahac = pow(pc_pi2 * pc_me * pc_kb * T / (pc_h * pc_h), 1.5);
  const double s = 2.0 / (y * D) * sahac;
  // stage fractions at the converged nelec, from log-weights phi_k
  double f[EOS_MAXST], E[EOS_MAXST];
  double pmax = 0.0;
  if (act) {
    f[0] = 0.0;
    E[0] = 0.0;
    for (int k = 1; k < nion; ++k) {
      f[k] = f[k - 1] + log(s) - e[k - 1] / kt + log(q[k]) - log(q[k - 1]);
      E[k] = E[k - 1] + e[k - 1];
      pmax = fmax(pmax, f[k]);
    }
  }
  double zs = 0.0;
  for (int k = 0; k < nion; ++k) zs += exp(f[k] - pmax);
  double ne = 0.0, me = 0.0;  // <k>, <E_k> over the stages
  for (int k = 0; k < nion; ++k) {
    f[k] = exp(f[k] - pmax) / zs;
    ne += (double)k * f[k];
    me += E[k] * f[k];
  }
  double V = 0.0, Cv = 0.0;
  for (int k = 0; k < nion; ++k) {
    V += f[k] * sq((double)k - ne);
    Cv += f[k] * ((double)k - ne) * (E[k] - me);
  }
  Cv = Cv / (kt * T);
  // oc_k = D fr (g1/q)_k f_k
  double gD = 0.0, gfr_l = 0.0, gbar = 0.0;
  double gf[EOS_MAXST];
  for (int k = 0; k < nion; ++k) {
    gf[k] = 0.0;
    if (k < A.noc) {
      const double go = goc[(size_t)i + (size_t)A.nc * ((size_t)k + (size_t)A.noc * lane)];
      const double w = g1[k] / q[k];
      gD += go * fr * w * f[k];
      gfr_l += go * D * w * f[k];
      gf[k] = go * D * fr * w;
    }
    gbar += gf[k] * f[k];
  }
  // through the normalisation: dL/dphi_k = f_k (gf_k - gbar); phi_k = k ln s + E_k/kT + const
  double glns = 0.0, gt = 0.0;
  for (int k = 0; k < nion; ++k) {
    const double gp = f[k] * (gf[k] - gbar);
    glns += gp * (double)k;
    gt += gp * E[k] / (kt * T);
  }
  // warp sums of the terms every element shares (nelec, T, D)
  double Gy = fr * V, GT = fr * (V * 1.5 / T + Cv), GD = fr * V;
  for (int o = 16; o > 0; o >>= 1) {
    glns += __shfl_xor_sync(0xffffffffu, glns, o);
    gt += __shfl_xor_sync(0xffffffffu, gt, o);
    gD += __shfl_xor_sync(0xffffffffu, gD, o);
    Gy += __shfl_xor_sync(0xffffffffu, Gy, o);
    GT += __shfl_xor_sync(0xffffffffu, GT, o);
    GD += __shfl_xor_sync(0xffffffffu, GD, o);
  }
  // ln s = ln(2 sahac(T)) - ln nelec - ln D
  gt += glns * 1.5 / T;
  const double gy = gnelec[i] - glns / y;
  gD += -glns / D;
  // nelec = G(nelec, T, D, fr) with dG/dnelec = -Gy/nelec, dG/dD = -GD/D
  const double lam = gy / (1.0 + Gy / y);
  gt += lam * GT;
  gD += lam * (-GD / D);
  if (act) gfr[(size_t)i * (A.nelem + 1) + lane + 1] += gfr_l + lam * ne;
  if (lane == 0) {
    gT[i] += gt;
    gnatom[i] += gD / vol;
  }
}

// massfr2natomfr (GAS/gas_setup.f:101-160) for differentiable inputs: mass
// fractions X (nelem, ncell) renormalised to one, gas_mass = rho vol,
// natomfr(z) ~ X_z/m_z normalised, gas_natom = mass sum(X/m) / amu.
__global__ void composition_kernel(int nc, int nelem, const double* __restrict__ rho, const double* __restrict__ X,
                                   const double* __restrict__ vol, const double* __restrict__ amass,
                                   double* __restrict__ mass, double* __restrict__ natom,
                                   double* __restrict__ natomfr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nc) return;
  const double* x = X + (size_t)i * nelem;
  double sx = 0.0;
  for (int z = 0; z < nelem; ++z) sx += x[z];
  double S = 0.0;
  for (int z = 0; z < nelem; ++z) S += (x[z] / sx) / amass[z];
  const double m = rho[i] * vol[i];
  mass[i] = m;
  natom[i] = m * S / pc_amu;
  double* fr = natomfr + (size_t)i * (nelem + 1);
  fr[0] = 0.0;
  for (int z = 0; z < nelem; ++z) fr[z + 1] = ((x[z] / sx) / amass[z]) / S;
}

// Adjoint of composition_kernel: gnatom, gfr -> grho, gX.
__global__ void composition_bwd_kernel(int nc, int nelem, const double* __restrict__ rho,
                                       const double* __restrict__ X, const double* __restrict__ vol,
                                       const double* __restrict__ amass, const double* __restrict__ gnatom,
                                       const double* __restrict__ gfr, double* __restrict__ grho,
                                       double* __restrict__ gX) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nc) return;
  const double* x = X + (size_t)i * nelem;
  const double* g = gfr + (size_t)i * (nelem + 1);
  double sx = 0.0;
  for (int z = 0; z < nelem; ++z) sx += x[z];
  double S = 0.0, gy_fr = 0.0;
  for (int z = 0; z < nelem; ++z) S += (x[z] / sx) / amass[z];
  for (int z = 0; z < nelem; ++z) gy_fr += g[z + 1] * ((x[z] / sx) / amass[z]);
  const double m = rho[i] * vol[i];
  grho[i] = gnatom[i] * vol[i] * S / pc_amu;
  // y_z = Xhat_z/m_z, S = sum y, natom = m S/amu, fr_z = y_z/S
  const double gS = gnatom[i] * m / pc_amu - gy_fr / (S * S);
  double dot = 0.0;
  double* gx = gX + (size_t)i * nelem;
  for (int z = 0; z < nelem; ++z) {
    const double gxh = (g[z + 1] / S + gS) / amass[z];
    gx[z] = gxh;
    dot += gxh * (x[z] / sx);
  }
  for (int z = 0; z < nelem; ++z) gx[z] = (gx[z] - dot) / sx;  // Xhat = X / sum X
}

int launch_saha_eos(slg_ctx* ctx, const double* temp, const double* natom, const double* vol,
                    const double* natomfr, double acc, double* nelec, int noc, double* oc, double* ginv,
                    int32_t* iconv, int* d_flags) {
  EosArgs A{ctx->nx, ctx->eos_nelem, ctx->eos_nstage, noc, ctx->d_eos_ni, ctx->d_eos_e, ctx->d_eos_q,
            ctx->d_eos_g1, temp, natom, vol, natomfr, acc, nelec, oc, ginv, iconv, d_flags};
  const long long nthr = (long long)ctx->nx * 32;
  saha_eos_kernel<<<(unsigned)((nthr + EOS_BLOCK - 1) / EOS_BLOCK), EOS_BLOCK, 0, ctx->stream>>>(A);
  return cuda_check(ctx, cudaGetLastError(), "saha_eos launch");
}

int check_eos(slg_ctx* ctx, int noc) {
  if (ctx->eos_nelem < 1) return set_error(ctx, SLG_ERR_STATE, "ion data not set (slg_set_ions)");
  if (ctx->nx < 1) return set_error(ctx, SLG_ERR_STATE, "grid not set");
  if (noc < 1) return set_error(ctx, SLG_ERR_ARG, "noc < 1");
  return SLG_OK;
}

}  // namespace

// Launchers used by the differentiable opacity (adjoint.cu).
int launch_composition(slg_ctx* ctx, const double* rho, const double* X, double* mass, double* natom,
                       double* natomfr) {
  const int nc = ctx->nx;
  composition_kernel<<<(nc + 127) / 128, 128, 0, ctx->stream>>>(nc, ctx->eos_nelem, rho, X, ctx->d_vol,
                                                                ctx->d_amass, mass, natom, natomfr);
  return cuda_check(ctx, cudaGetLastError(), "composition launch");
}

int launch_composition_bwd(slg_ctx* ctx, const double* rho, const double* X, const double* gnatom,
                           const double* gfr, double* grho, double* gX) {
  const int nc = ctx->nx;
  composition_bwd_kernel<<<(nc + 127) / 128, 128, 0, ctx->stream>>>(nc, ctx->eos_nelem, rho, X, ctx->d_vol,
                                                                    ctx->d_amass, gnatom, gfr, grho, gX);
  return cuda_check(ctx, cudaGetLastError(), "composition adjoint launch");
}

int launch_saha_eos_dev(slg_ctx* ctx, const double* temp, const double* natom, const double* vol,
                        const double* natomfr, double acc, double* nelec, int noc, double* oc, double* ginv,
                        int* d_flags) {
  return launch_saha_eos(ctx, temp, natom, vol, natomfr, acc, nelec, noc, oc, ginv, nullptr, d_flags);
}

int launch_saha_eos_bwd(slg_ctx* ctx, const double* temp, const double* natom, const double* vol,
                        const double* natomfr, const double* nelec, int noc, const double* goc,
                        const double* gnelec, double* gT, double* gnatom, double* gfr) {
  EosArgs A{ctx->nx, ctx->eos_nelem, ctx->eos_nstage, noc, ctx->d_eos_ni, ctx->d_eos_e, ctx->d_eos_q,
            ctx->d_eos_g1, temp, natom, vol, natomfr, 0.0, const_cast<double*>(nelec), nullptr, nullptr,
            nullptr, nullptr};
  const long long nthr = (long long)ctx->nx * 32;
  saha_eos_bwd_kernel<<<(unsigned)((nthr + EOS_BLOCK - 1) / EOS_BLOCK), EOS_BLOCK, 0, ctx->stream>>>(
      A, goc, gnelec, gT, gnatom, gfr);
  return cuda_check(ctx, cudaGetLastError(), "saha_eos adjoint launch");
}

}  // namespace slg

using namespace slg;

extern "C" {

void slg_partition_functions(int32_t nelem, int32_t nstage, int32_t nlev, const int32_t* ni, const int32_t* nlevel,
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

int slg_set_ions(slg_ctx* ctx, int32_t nelem, int32_t nstage, const int32_t* ni, const double* e, const double* q,
                 const double* g1) {
  if (!ctx || nelem < 1 || nelem > 32 || nstage < 2 || nstage > EOS_MAXST || !ni || !e || !q || !g1)
    return set_error(ctx, SLG_ERR_ARG, "slg_set_ions: bad arguments (1 <= nelem <= 32, 2 <= nstage <= 32)");
  for (int iz = 0; iz < nelem; ++iz) {
    if (ni[iz] < 1 || ni[iz] > nstage) return set_error(ctx, SLG_ERR_ARG, "slg_set_ions: ni(%d) = %d", iz + 1, ni[iz]);
    for (int ii = 0; ii < ni[iz]; ++ii)
      if (!(q[(size_t)iz * nstage + ii] > 0.0) || !(g1[(size_t)iz * nstage + ii] > 0.0))
        return set_error(ctx, SLG_ERR_ARG, "slg_set_ions: q or g1 of ion (%d,%d) not positive", iz + 1, ii + 1);
  }
  cudaSetDevice(ctx->device);
  const size_t n = (size_t)nelem * nstage;
  if (ctx->eos_nelem != nelem || ctx->eos_nstage != nstage) {
    cudaFree(ctx->d_eos_ni); cudaFree(ctx->d_eos_e); cudaFree(ctx->d_eos_q); cudaFree(ctx->d_eos_g1);
    ctx->d_eos_ni = nullptr; ctx->d_eos_e = ctx->d_eos_q = ctx->d_eos_g1 = nullptr;
    ctx->eos_nelem = ctx->eos_nstage = 0;
    int rc = cuda_check(ctx, cudaMalloc(&ctx->d_eos_ni, sizeof(int32_t) * nelem), "alloc ions");
    if (!rc) rc = cuda_check(ctx, cudaMalloc(&ctx->d_eos_e, sizeof(double) * n), "alloc ions");
    if (!rc) rc = cuda_check(ctx, cudaMalloc(&ctx->d_eos_q, sizeof(double) * n), "alloc ions");
    if (!rc) rc = cuda_check(ctx, cudaMalloc(&ctx->d_eos_g1, sizeof(double) * n), "alloc ions");
    if (rc) return rc;
  }
  int rc = cuda_check(ctx, cudaMemcpy(ctx->d_eos_ni, ni, sizeof(int32_t) * nelem, cudaMemcpyHostToDevice), "ions");
  if (!rc) rc = cuda_check(ctx, cudaMemcpy(ctx->d_eos_e, e, sizeof(double) * n, cudaMemcpyHostToDevice), "ions");
  if (!rc) rc = cuda_check(ctx, cudaMemcpy(ctx->d_eos_q, q, sizeof(double) * n, cudaMemcpyHostToDevice), "ions");
  if (!rc) rc = cuda_check(ctx, cudaMemcpy(ctx->d_eos_g1, g1, sizeof(double) * n, cudaMemcpyHostToDevice), "ions");
  if (rc) return rc;
  ctx->eos_nelem = nelem;
  ctx->eos_nstage = nstage;
  return SLG_OK;
}

int slg_dev_saha_eos(slg_ctx* ctx, const double* temp, const double* natom, const double* vol, const double* natomfr,
                     double acc, double* nelec, int32_t noc, double* oc, double* ginv, int32_t* iconv) {
  if (!ctx || !temp || !natom || !vol || !natomfr || !nelec || !oc || !ginv || !(acc > 0.0))
    return set_error(ctx, SLG_ERR_ARG, "slg_dev_saha_eos: bad arguments");
  int rc = check_eos(ctx, noc);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  int* d_flags = (int*)scratch(ctx, 50, sizeof(int) * 2);
  if (!d_flags) return SLG_ERR_OOM;
  cudaMemsetAsync(d_flags, 0, sizeof(int) * 2, ctx->stream);
  return launch_saha_eos(ctx, temp, natom, vol, natomfr, acc, nelec, noc, oc, ginv, iconv, d_flags);
}

int slg_saha_eos(slg_ctx* ctx, const double* temp, const double* natom, const double* vol, const double* natomfr,
                 double acc, double* nelec, int32_t noc, double* oc, double* ginv, int32_t* iconv) {
  if (!ctx || !temp || !natom || !vol || !natomfr || !nelec || !oc || !ginv || !(acc > 0.0))
    return set_error(ctx, SLG_ERR_ARG, "slg_saha_eos: bad arguments");
  int rc = check_eos(ctx, noc);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  const size_t nc = ctx->nx, nfr = nc * (ctx->eos_nelem + 1), noct = nc * noc * ctx->eos_nelem;
  double* d = (double*)scratch(ctx, 51, sizeof(double) * (3 * nc + nfr + nc + 2 * noct));
  int* d_flags = (int*)scratch(ctx, 50, sizeof(int) * 2);
  int32_t* d_it = (int32_t*)scratch(ctx, 52, sizeof(int32_t) * nc);
  if (!d || !d_flags || !d_it) return SLG_ERR_OOM;
  double *dt = d, *dna = d + nc, *dv = d + 2 * nc, *dfr = d + 3 * nc, *dne = dfr + nfr, *doc = dne + nc,
         *dgi = doc + noct;
  cudaStream_t st = ctx->stream;
  rc = cuda_check(ctx, cudaMemcpyAsync(dt, temp, sizeof(double) * nc, cudaMemcpyHostToDevice, st), "eos in");
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(dna, natom, sizeof(double) * nc, cudaMemcpyHostToDevice, st), "eos in");
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(dv, vol, sizeof(double) * nc, cudaMemcpyHostToDevice, st), "eos in");
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(dfr, natomfr, sizeof(double) * nfr, cudaMemcpyHostToDevice, st), "eos in");
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(dne, nelec, sizeof(double) * nc, cudaMemcpyHostToDevice, st), "eos in");
  if (rc) return rc;
  cudaMemsetAsync(d_flags, 0, sizeof(int) * 2, st);
  rc = launch_saha_eos(ctx, dt, dna, dv, dfr, acc, dne, noc, doc, dgi, d_it, d_flags);
  int h_flags = 0;
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(nelec, dne, sizeof(double) * nc, cudaMemcpyDeviceToHost, st), "eos out");
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(oc, doc, sizeof(double) * noct, cudaMemcpyDeviceToHost, st), "eos out");
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(ginv, dgi, sizeof(double) * noct, cudaMemcpyDeviceToHost, st), "eos out");
  if (!rc && iconv)
    rc = cuda_check(ctx, cudaMemcpyAsync(iconv, d_it, sizeof(int32_t) * nc, cudaMemcpyDeviceToHost, st), "eos out");
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(&h_flags, d_flags, sizeof(int), cudaMemcpyDeviceToHost, st), "eos out");
  const int rs = cuda_check(ctx, cudaStreamSynchronize(st), "eos sync");
  if (rc) return rc;
  if (rs) return rs;
  if (h_flags & 1) return set_error(ctx, SLG_ERR_ARG, "saha_eos: a cell where ions_solve_eos stops (invalid sum or nelec <= 0)");
  return SLG_OK;
}

}  // extern "C"
