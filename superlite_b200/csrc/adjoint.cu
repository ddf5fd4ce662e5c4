// adjoint.cu -- the opacity build as a differentiable function of shell
// temperature, density and mass fractions, with its hand-written reverse mode
// (no counterpart in the reference, which only runs the forward build).
//
// Forward:  massfr2natomfr (GAS/gas_setup.f:101-160) -> ions_solve_eos +
//           eos_update (ionsmod.f:160-356, GAS/eos_update.f:20-45) ->
//           physical_opacity (GAS/physical_opacity.f, ngs = 1, FP64 result) ->
//           opacity_planckmean / opacity_rossmean and leakage_opacity11 on
//           the FP64 opacity.
// Reverse:  the adjoints of those stages in the opposite order; every
//           per-cell stage is local to the cell except leakage_opacity11,
//           whose adjoint also feeds the neighbouring shells.
// The equation of state is solved to the caller's accuracy (1e-14 keeps the
// forward smooth enough for finite differences); its adjoint is the implicit
// derivative at that solution.
#include <cuda_runtime.h>
#include "slg_device.cuh"
#include "slg_internal.h"

namespace slg {
int launch_composition(slg_ctx* ctx, const double* rho, const double* X, double* mass, double* natom,
                       double* natomfr);
int launch_composition_bwd(slg_ctx* ctx, const double* rho, const double* X, const double* gnatom,
                           const double* gfr, double* grho, double* gX);
int launch_saha_eos_dev(slg_ctx* ctx, const double* temp, const double* natom, const double* vol,
                        const double* natomfr, double acc, double* nelec, int noc, double* oc, double* ginv,
                        int* d_flags);
int launch_saha_eos_bwd(slg_ctx* ctx, const double* temp, const double* natom, const double* vol,
                        const double* natomfr, const double* nelec, int noc, const double* goc,
                        const double* gnelec, double* gT, double* gnatom, double* gfr);
int launch_physical_opacity64(slg_ctx* ctx, const slg_gas* gas, double* gas_sig, double* capg64, float* gas_cap,
                              float* gas_emiss);
int launch_opacity_means64(slg_ctx* ctx, const double* temp, const double* sig, const double* cap,
                           double* capgrey, double* capross);
int launch_means_bwd(slg_ctx* ctx, const double* temp, const double* sig, const double* cap, const double* capross,
                     const double* ggrey, const double* gross, double* gcap, double* gsig, double* gT);
int launch_opacity_bwd(slg_ctx* ctx, const slg_gas* gas, const double* gcap, const double* gsig, double* gT,
                       double* goc, double* gnelec, double* gnatom, double* gfr, double* sig_work, double* work);
int launch_leakage64(slg_ctx* ctx, const double* tempinv, const double* sig, const double* cap, double tauddmc,
                     double taulump, double* opaclump);
int launch_leakage64_bwd(slg_ctx* ctx, const double* tempinv, const double* sig, const double* cap,
                         double tauddmc, double taulump, const double* opaclump, const double* gol, double* gcap,
                         double* gsig, double* gT);

namespace {

__global__ void reciprocal_kernel(int n, const double* __restrict__ a, double* __restrict__ r) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = 1.0 / a[i];
}

// Gas state of the forward for given inputs (scratch slots 53..61); the
// reverse mode works in slots 64..71.
struct GasState {
  double *mass, *natom, *natomfr, *oc, *ginv, *tempinv, *nelec;
  int* flags;
  slg_gas gas;
};

int check_ready(slg_ctx* ctx) {
  if (ctx->nx < 1 || ctx->ng < 1) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  if (ctx->nelem < 1) return set_error(ctx, SLG_ERR_STATE, "atomic data not set");
  if (ctx->eos_nelem != ctx->nelem)
    return set_error(ctx, SLG_ERR_STATE, "ion data (slg_set_ions) not set for the atomic data's elements");
  if (ctx->amass_n != ctx->nelem) return set_error(ctx, SLG_ERR_STATE, "element masses not set");
  if (ctx->nmodel > 1) return set_error(ctx, SLG_ERR_STATE, "the differentiable opacity takes one model");
  return SLG_OK;
}

// composition + equation of state, starting from nelec_in
int gas_state(slg_ctx* ctx, const double* temp, const double* rho, const double* massfr, double acc,
              const double* nelec_in, GasState& S) {
  const int nc = ctx->nx, nel = ctx->nelem, nst = ctx->nstage;
  const size_t nocn = (size_t)nc * nst * nel;
  S.mass = (double*)scratch(ctx, 53, sizeof(double) * nc);
  S.natom = (double*)scratch(ctx, 54, sizeof(double) * nc);
  S.natomfr = (double*)scratch(ctx, 55, sizeof(double) * nc * (nel + 1));
  S.oc = (double*)scratch(ctx, 56, sizeof(double) * nocn);
  S.ginv = (double*)scratch(ctx, 57, sizeof(double) * nocn);
  S.tempinv = (double*)scratch(ctx, 58, sizeof(double) * nc);
  S.nelec = (double*)scratch(ctx, 59, sizeof(double) * nc);
  S.flags = (int*)scratch(ctx, 61, sizeof(int) * 2);
  if (!S.mass || !S.natom || !S.natomfr || !S.oc || !S.ginv || !S.tempinv || !S.nelec || !S.flags)
    return SLG_ERR_OOM;
  cudaStream_t st = ctx->stream;
  cudaMemsetAsync(S.flags, 0, sizeof(int) * 2, st);
  cudaMemcpyAsync(S.nelec, nelec_in, sizeof(double) * nc, cudaMemcpyDeviceToDevice, st);
  int rc = launch_composition(ctx, rho, massfr, S.mass, S.natom, S.natomfr);
  if (!rc) rc = launch_saha_eos_dev(ctx, temp, S.natom, ctx->d_vol, S.natomfr, acc, S.nelec, nst, S.oc, S.ginv,
                                    S.flags);
  reciprocal_kernel<<<(nc + 127) / 128, 128, 0, st>>>(nc, temp, S.tempinv);
  S.gas = slg_gas{temp, S.natom, S.nelec, ctx->d_vol, S.mass, S.natomfr, S.oc, S.ginv};
  return rc ? rc : cuda_check(ctx, cudaGetLastError(), "gas state");
}

}  // namespace
}  // namespace slg

using namespace slg;

extern "C" {

int slg_set_element_masses(slg_ctx* ctx, int32_t nelem, const double* mass_amu) {
  if (!ctx || nelem < 1 || !mass_amu) return set_error(ctx, SLG_ERR_ARG, "slg_set_element_masses: bad arguments");
  for (int z = 0; z < nelem; ++z)
    if (!(mass_amu[z] > 0.0)) return set_error(ctx, SLG_ERR_ARG, "element %d: mass not positive", z + 1);
  cudaSetDevice(ctx->device);
  if (ctx->amass_n != nelem) {
    cudaFree(ctx->d_amass);
    ctx->d_amass = nullptr;
    ctx->amass_n = 0;
    const int rc = cuda_check(ctx, cudaMalloc(&ctx->d_amass, sizeof(double) * nelem), "alloc masses");
    if (rc) return rc;
  }
  const int rc = cuda_check(ctx, cudaMemcpy(ctx->d_amass, mass_amu, sizeof(double) * nelem, cudaMemcpyHostToDevice),
                            "masses");
  if (!rc) ctx->amass_n = nelem;
  return rc;
}

int slg_dev_opacity_grad_forward(slg_ctx* ctx, const double* temp, const double* rho, const double* massfr,
                                 double acc, double tauddmc, double taulump, double* nelec, double* cap, double* sig,
                                 double* capgrey, double* capross, double* opaclump) {
  if (!ctx || !temp || !rho || !massfr || !nelec || !cap || !sig || !capgrey || !capross || !opaclump || !(acc > 0.0))
    return set_error(ctx, SLG_ERR_ARG, "slg_dev_opacity_grad_forward: bad arguments");
  int rc = check_ready(ctx);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  const size_t ncg = (size_t)ctx->nx * ctx->ng;
  float* c32 = (float*)scratch(ctx, 62, sizeof(float) * ncg);
  float* e32 = (float*)scratch(ctx, 63, sizeof(float) * ncg);
  if (!c32 || !e32) return SLG_ERR_OOM;
  GasState S;
  rc = gas_state(ctx, temp, rho, massfr, acc, nelec, S);
  if (!rc) rc = launch_physical_opacity64(ctx, &S.gas, sig, cap, c32, e32);
  if (!rc) rc = launch_opacity_means64(ctx, temp, sig, cap, capgrey, capross);
  if (!rc) rc = launch_leakage64(ctx, S.tempinv, sig, cap, tauddmc, taulump, opaclump);
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(nelec, S.nelec, sizeof(double) * ctx->nx, cudaMemcpyDeviceToDevice,
                                                ctx->stream), "nelec");
  return rc;
}

int slg_dev_opacity_grad_backward(slg_ctx* ctx, const double* temp, const double* rho, const double* massfr,
                                  double acc, double tauddmc, double taulump, const double* nelec, const double* cap,
                                  const double* sig, const double* capgrey, const double* capross,
                                  const double* opaclump, const double* gcap, const double* gsig,
                                  const double* gcapgrey, const double* gcapross, const double* gopaclump,
                                  double* gtemp, double* grho, double* gmassfr) {
  (void)capgrey;
  if (!ctx || !temp || !rho || !massfr || !nelec || !cap || !sig || !capross || !opaclump || !gtemp || !grho ||
      !gmassfr || !(acc > 0.0))
    return set_error(ctx, SLG_ERR_ARG, "slg_dev_opacity_grad_backward: bad arguments");
  int rc = check_ready(ctx);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  const int nc = ctx->nx, ng = ctx->ng, nel = ctx->nelem, nst = ctx->nstage;
  const size_t nslot = (size_t)nel * nst;
  cudaStream_t st = ctx->stream;
  double* G = (double*)scratch(ctx, 64, sizeof(double) * (size_t)nc * ng);
  double* Gs = (double*)scratch(ctx, 65, sizeof(double) * nc);
  double* goc = (double*)scratch(ctx, 66, sizeof(double) * nslot * nc);
  double* gnel = (double*)scratch(ctx, 67, sizeof(double) * nc);
  double* gnat = (double*)scratch(ctx, 68, sizeof(double) * nc);
  double* gfr = (double*)scratch(ctx, 69, sizeof(double) * (size_t)nc * (nel + 1));
  double* sigw = (double*)scratch(ctx, 70, sizeof(double) * nc);
  double* work = (double*)scratch(ctx, 71, sizeof(double) * (nslot * nc + nc));
  if (!G || !Gs || !goc || !gnel || !gnat || !gfr || !sigw || !work) return SLG_ERR_OOM;
  GasState S;
  rc = gas_state(ctx, temp, rho, massfr, acc, nelec, S);
  if (rc) return rc;
  if (gcap) cudaMemcpyAsync(G, gcap, sizeof(double) * (size_t)nc * ng, cudaMemcpyDeviceToDevice, st);
  else cudaMemsetAsync(G, 0, sizeof(double) * (size_t)nc * ng, st);
  if (gsig) cudaMemcpyAsync(Gs, gsig, sizeof(double) * nc, cudaMemcpyDeviceToDevice, st);
  else cudaMemsetAsync(Gs, 0, sizeof(double) * nc, st);
  cudaMemsetAsync(gtemp, 0, sizeof(double) * nc, st);
  if (gcapgrey || gcapross) rc = launch_means_bwd(ctx, temp, sig, cap, capross, gcapgrey, gcapross, G, Gs, gtemp);
  if (!rc && gopaclump)
    rc = launch_leakage64_bwd(ctx, S.tempinv, sig, cap, tauddmc, taulump, opaclump, gopaclump, G, Gs, gtemp);
  if (!rc) rc = launch_opacity_bwd(ctx, &S.gas, G, Gs, gtemp, goc, gnel, gnat, gfr, sigw, work);
  if (!rc) rc = launch_saha_eos_bwd(ctx, temp, S.natom, ctx->d_vol, S.natomfr, S.nelec, nst, goc, gnel, gtemp, gnat,
                                    gfr);
  if (!rc) rc = launch_composition_bwd(ctx, rho, massfr, gnat, gfr, grho, gmassfr);
  return rc;
}

}  // extern "C"
