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
  // guide tables of the four running sums above (dop, left, right, scat):
  // per cell and table guide_m+1 entries, entry k = number of sums <= k/guide_m,
  // so a draw r in [k, k+1)/guide_m is searched only between entries k and k+1
  // (null: plain search over the whole table).  guide_m is a power of two
  // (so r * guide_m and k / guide_m are exact) near ng/4: a range of a few
  // entries, searched in one round of loads, without a guide larger than the
  // tables it indexes.
  int16_t* guide = nullptr;
  int guide_m = 0;
  // FP32 copies of cdf_dop/left/right/scat for the mixed-precision loop (half
  // the bytes per gather; null when only the FP64 loop runs)
  float *cdf32_dop = nullptr, *cdf32_left = nullptr, *cdf32_right = nullptr, *cdf32_scat = nullptr;
  int nx = 0, ng = 0;
};
constexpr int kGuideMax = 256;
inline int guide_size(int ng) {
  int m = 16;
  while (m < kGuideMax && 4 * m < ng) m *= 2;
  return m;
}

// Per-cell record of the mixed-precision particle loop: everything an event
// reads about its shell except per-group values, in one 128-byte line
// (instead of about ten lines of separate arrays).  Values are the same
// roundings the event code made from the separate arrays.
struct alignas(128) MixCell {
  double xa, xb, vxa, vxb;  // shell edges and edge velocities
  double x0;                // the model's inner edge
  double capgreyinv, tinv;  // 1/capgrey, 1/T
  int nlump, pad;
  float dist, sig, emitlump, caplump, doplump, o1, o2, divv;  // o1, o2: opaclump(1:2) of the lumped groups
  float far, dvdr, sigl, sigr, dxl, dxr, fa, fb;  // neighbours (0 at the model's ends); fa, fb = x^2 / dx3
};
static_assert(sizeof(MixCell) == 128, "MixCell is one 128-byte line");
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

// One ejecta model of a multi-model context: particle slots [poff, poff+np),
// cells [co, co+nx) of every per-cell array, shell edges [xo, xo+nx] of
// xarr/vxarr (xo = co + model index).
struct ModelDesc {
  long long poff, np;
  int nx, co, xo, pad;
};

// Random-number key of model m: seed + m * kModelSeedStride (SLG_MODEL_SEED_STRIDE).
constexpr unsigned long long kModelSeedStride = 0x9E3779B97F4A7C15ULL;

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
  // population rows (slot = (iz-1) nstage + ii-1) that the lines reference:
  // d_lrow_of_slot[slot] = compact row or -1, d_slot_of_lrow[row] = slot
  int nlrow = 0;
  double line_chimax = 0.0;  // largest chilw of the lines (infinite if any is negative or NaN)
  int16_t* d_lrow_of_slot = nullptr;
  int16_t* d_slot_of_lrow = nullptr;
  float* d_ph1 = nullptr;
  float* d_ph2 = nullptr;
  double* d_gff = nullptr;
  std::vector<float> h_ph1, h_ph2;
  // ion data of the equation of state: stages, ionisation energies,
  // partition functions and ground-level weights, (nstage, nelem) each
  int eos_nelem = 0, eos_nstage = 0;
  int32_t* d_eos_ni = nullptr;
  double* d_eos_e = nullptr;
  double* d_eos_q = nullptr;
  double* d_eos_g1 = nullptr;
  double* d_amass = nullptr;  // element masses [amu] of the differentiable opacity
  int amass_n = 0;
  // derived per-call scratch
  slg::DevBuf scratch[96];
  slg::CellTables tables;
  slg::TransportAcc* d_acc = nullptr;
  slg::TransportAcc* h_acc = nullptr;  // pinned
  // optional trace (host arrays) for the next particle_advance call
  uint64_t* trace_hash = nullptr;
  int32_t* trace_nstep = nullptr;
  // transport kernel variants until slg_autotune_transport or
  // slg_set_transport_variant choose: the ones measured fastest on whole
  // steps of the batched 128-model workload at full particle budgets
  int trn_variant = 2;  // FP64 transport kernel variant (see launch_transport_variant)
  int mix_variant = 3;  // mixed-precision variant (see launch_transport_mixed)
  // transport_out of a queued slg_dev_particle_advance, completed by slg_sync
  slg_transport_out* pending_out = nullptr;
  // models (one for slg_set_grid): host descriptors, device copies, and the
  // per-cell map {local 1-based shell, model nx, model first cell, model}
  int nmodel = 0;
  std::vector<slg::ModelDesc> h_models;
  slg::ModelDesc* d_models = nullptr;
  int4* d_cellmap = nullptr;  // null for a single model
  long long npart_models = 0;  // sum of the models' particle slots (0: one unranged model)
  // running sums of the transport counters over launches (device; they
  // survive graph replays), the replay counter that offsets the random
  // streams of captured launches, and the captured graph
  slg::TransportAcc* d_totals = nullptr;
  unsigned long long* d_epoch = nullptr;
  int capturing = 0;
  int capture_failed = 0;  // a call failed during the open capture
  cudaGraphExec_t graph_exec = nullptr;
  // host copies of the last uploaded source set-up (an unchanged set-up is
  // not uploaded again, so captured steps hold no host copies)
  std::vector<double> src_emit;
  std::vector<int32_t> src_nvol;
  int num_sms = 0;
};

namespace slg {
// Raises kernel `fn`'s dynamic shared-memory limit to `bytes` on the current
// device (the context's: every entry point selects it) the first time a
// launch there needs it; the attribute holds per device, so `mask` keeps one
// bit per device id.
template <class F>
inline void raise_smem_limit(unsigned& mask, int device, F* fn, int bytes) {
  const unsigned bit = device >= 0 && device < 32 ? 1u << device : 0u;
  if (bit && (mask & bit)) return;
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  mask |= bit;
}

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
