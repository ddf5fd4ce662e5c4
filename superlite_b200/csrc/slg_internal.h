// slg_internal.h -- host-side context and launch declarations of libslg.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>
#include "slg.h"

namespace slg {

// A device buffer that grows on demand and is freed with the context.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// Device-resident per-cell tables used by the transport kernels (built by
// build_cell_tables from grd_cap, grd_sig, grd_opaclump ...).  All tables
// are cell-major: entry (ic-1)*ng + k.
struct CellTables {
  double* specarr = nullptr;  // specintv mode-0 Planck weights
  int16_t* glumps = nullptr;  // diffusion11.f90:103-124 ordering (1-based groups)
  double* cdf_dop = nullptr;  // Doppler resolved-group partial sums (:290-314)
  double* cdf_left = nullptr; // left-leak resolved-group partial sums (:375-398)
  double* cdf_right = nullptr;// right-leak partial sums (:447-460 at ix==nx, :489-511 else)
  double* cdf_scat = nullptr; // effective-scatter partial sums over unlumped groups (:571-584)
  double* emitcum = nullptr;  // emitgroup within-bin running sums (emitgroup.f:311-320)
  // per-cell scalars: nlump, emitlump, caplump, doplump, capgreyinv, speclump
  int32_t* nlump = nullptr;
  double* scal = nullptr;     // 8 doubles per cell (see SCAL_*)
  int nx = 0, ng = 0;
};
enum { SCAL_EMITLUMP = 0, SCAL_CAPLUMP, SCAL_DOPLUMP, SCAL_CAPGREYINV, SCAL_SPECLUMP, SCAL_FAR,
       SCAL_DX3, SCAL_DVDR, SCAL_N };

// Accumulators written by the transport kernel (device memory).
struct TransportAcc {
  double evelo, eout, sflux;
  unsigned long long npckt, nflux, nimc, nddmc, nswap, nmax, nwarn;
  unsigned long long ndist[11];
  unsigned long long ierr_key;  // (ipart << 32) | ierr, min over particles
  unsigned long long next;      // persistent-kernel work counter
};

}  // namespace slg

struct slg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  // groups
  int ng = 0, nep = 0, nepg = 0;
  double* d_wl = nullptr;
  double* d_wlinv = nullptr;
  std::vector<double> h_wl;
  // grid
  int nx = 0;
  double* d_xarr = nullptr;
  double* d_vxarr = nullptr;
  double* d_vol = nullptr;
  double* d_divv = nullptr;
  std::vector<double> h_xarr;
  // atomic data
  int nelem = 0, nstage = 0;
  int64_t nline = 0;
  int32_t* d_ion_ni = nullptr;
  std::vector<int32_t> h_ion_ni;
  slg_bbxs* d_bb = nullptr;
  float* d_ph1 = nullptr;
  float* d_ph2 = nullptr;
  double* d_gff = nullptr;
  std::vector<float> h_ph1, h_ph2;
  // derived per-call scratch
  slg::DevBuf scratch[64];
  slg::CellTables tables;
  slg::TransportAcc* d_acc = nullptr;
  slg::TransportAcc* h_acc = nullptr;  // pinned
  // optional trace (host arrays) for the next particle_advance call
  uint64_t* trace_hash = nullptr;
  int32_t* trace_nstep = nullptr;
  // launch configuration chosen by the autotuner (0 = defaults)
  int trn_variant = 0;  // transport kernel variant (see launch_transport_variant)
  // transport_out of a queued slg_dev_particle_advance, completed by slg_sync
  slg_transport_out* pending_out = nullptr;
  int num_sms = 0;
};

namespace slg {
int set_error(slg_ctx* ctx, int code, const char* fmt, ...);
int cuda_check(slg_ctx* ctx, cudaError_t e, const char* what);
void* scratch(slg_ctx* ctx, int slot, size_t bytes);  // nullptr on failure (error set)

// kernels launch wrappers (return SLG_OK or error)
int launch_physical_opacity(slg_ctx* ctx, const slg_gas* gas, const slg_opacity_flags* flags,
                            double* gas_sig, float* gas_cap, float* gas_emiss, double* cap64);
int launch_analytic_opacity(slg_ctx* ctx, const double* temp, const double* rho, int kind,
                            const double* coefs, double* gas_sig, float* gas_cap);
int launch_opacity_means(slg_ctx* ctx, const double* temp, const double* sig, const float* cap,
                         double* capgrey, double* capross);
int launch_leakage(slg_ctx* ctx, const double* tempinv, const double* sig, const float* cap,
                   const float* capemit, double tauddmc, double taulump, double* opaclump);
int launch_emitprob(slg_ctx* ctx, const double* tempinv, const float* cap, const double* capgrey,
                    double* emitprob);
int build_cell_tables(slg_ctx* ctx, const slg_transport_in* in);
int launch_particle_advance(slg_ctx* ctx, const slg_transport_in* in, slg_packet* prt,
                            int32_t* isvacant, int64_t npart, uint64_t seed,
                            slg_transport_out* out, uint64_t* d_trace_hash, int32_t* d_trace_nstep);
int finish_particle_advance(slg_ctx* ctx, const slg_transport_in* in, slg_transport_out* out);
int launch_fluxtally(slg_ctx* ctx, int64_t npart, const slg_packet* prt, int32_t* isvacant,
                     int flx_ng, const double* flx_wl, double* luminos, double* lumdev,
                     int32_t* lumnum);
int launch_sourcetally(slg_ctx* ctx, int64_t npart, const slg_packet* prt, const int32_t* isvacant,
                       double* src_energy, int32_t* src_number);
}  // namespace slg
