// noalloc.cu -- particle_advance for callers that cannot allocate device memory.
//
// Some callers of this library run where they may not call cudaMalloc: a host
// code that hands every device buffer to the GPU from its own memory pool and
// forbids other allocations, a call made while another component owns the
// device allocator, or an embedding that budgets every byte of HBM up front.
// slg_particle_advance_static serves them: the caller passes every input and
// output as a device pointer, and the per-cell tables and counters that
// particle_advance needs live in one file-scope __device__ array of fixed size
// that every GPU loading the library holds until the process exits.
//
// Limits and sharing: the array holds the tables of at most
// SLG_STATIC_MAX_CELLGROUPS (ncell * ng) entries and SLG_STATIC_MAX_CELLS
// cells, with at most SLG_MAX_GROUPS groups (group lists are int16); larger
// grids are rejected with SLG_ERR_TOO_LARGE.  All calls share
// the one array and it keeps the last call's contents: counters are cleared at
// the start of every call, and calls that overlap on the GPU (two streams, two
// host threads) race on it.
#include <cuda_runtime.h>
#include <mutex>
#include "slg.h"
#include "slg_internal.h"
#include "transport_impl.cuh"

namespace slg {
int launch_cell_tables_raw(cudaStream_t st, int nx, int ng, int nep, int nepg, const double* xarr,
                           const double* vxarr, const double* divv, const double* wlinv,
                           const slg_transport_in* in, const CellTables& T);
int launch_particle_advance_raw(cudaStream_t st, const TrnArgs& A, int nblk);
int particle_advance_blocks_per_sm();
int particle_advance_block_size();
int finish_particle_advance_acc(const TransportAcc& a, slg_transport_out* out);
}  // namespace slg

namespace {

constexpr size_t kMaxCellGroups = SLG_STATIC_MAX_CELLGROUPS;
constexpr size_t kMaxCells = SLG_STATIC_MAX_CELLS;
constexpr size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
// layout of the array: accumulators, per-cell scalars, then the (ncell, ng) tables
constexpr size_t kAccBytes = align256(sizeof(slg::TransportAcc));
constexpr size_t kNlumpBytes = align256(sizeof(int32_t) * kMaxCells);
constexpr size_t kScalBytes = align256(sizeof(double) * slg::SCAL_N * kMaxCells);
constexpr size_t kTabBytes = align256(sizeof(double) * kMaxCellGroups);
constexpr size_t kGlumpBytes = align256(sizeof(int16_t) * kMaxCellGroups);
constexpr size_t kScratchBytes = kAccBytes + kNlumpBytes + kScalBytes + 6 * kTabBytes + kGlumpBytes;

static __device__ __align__(256) unsigned char g_static_scratch[kScratchBytes];

// Device address of g_static_scratch, per device ordinal (host code must not
// use the symbol itself as an address).
constexpr int kMaxDevices = 64;
unsigned char* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_setup_mutex;

int scratch_address(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices) return SLG_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p) return SLG_ERR_CUDA;
    g_scratch_addr[dev] = (unsigned char*)p;
  }
  *out = g_scratch_addr[dev];
  return SLG_OK;
}

}  // namespace

extern "C" int slg_particle_advance_static(const slg_grid_dev* grid, const slg_transport_in* in,
                                           slg_packet* prt, int32_t* isvacant, int64_t npart,
                                           uint64_t seed, slg_transport_out* out, void* stream) {
  using namespace slg;
  if (!grid || !in || !out || npart < 0 || (npart > 0 && (!prt || !isvacant))) return SLG_ERR_ARG;
  if (!grid->xarr || !grid->vxarr || !grid->divv || !grid->wl || !grid->wlinv || grid->nx < 2 || grid->ng < 1)
    return SLG_ERR_ARG;
  if (!in->tempinv || !in->sig || !in->capgrey || !in->emitprob || !in->opaclump || !in->cap) return SLG_ERR_ARG;
  if (!out->tally || !out->jrad || !out->eamp || (in->dogrdtally && !out->methodswap)) return SLG_ERR_ARG;
  if (in->precision != 0) return SLG_ERR_NOT_BUILT;
  const size_t nx = (size_t)grid->nx, ng = (size_t)grid->ng;
  if (nx > kMaxCells || nx * ng > kMaxCellGroups || ng > SLG_MAX_GROUPS) return SLG_ERR_TOO_LARGE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SLG_ERR_CUDA;
  unsigned char* base = nullptr;
  int rc = scratch_address(dev, &base);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // carve the static array
  TransportAcc* acc = (TransportAcc*)base;
  unsigned char* p = base + kAccBytes;
  CellTables T;
  T.nlump = (int32_t*)p;
  p += kNlumpBytes;
  T.scal = (double*)p;
  p += kScalBytes;
  double* tabs[6];
  for (int k = 0; k < 6; ++k) {
    tabs[k] = (double*)p;
    p += kTabBytes;
  }
  T.specarr = tabs[0];
  T.cdf_dop = tabs[1];
  T.cdf_left = tabs[2];
  T.cdf_right = tabs[3];
  T.cdf_scat = tabs[4];
  T.emitcum = tabs[5];
  T.glumps = (int16_t*)p;
  T.nx = (int)nx;
  T.ng = (int)ng;
  const int nep = (int)lround(std::sqrt((double)ng));          // gridmod.f:121
  const int nepg = (int)std::ceil((double)ng / (nep + 1.0));     // gridmod.f:122
  // clear what must start at zero: the counters and the tallies
  if (cudaMemsetAsync(acc, 0, sizeof(TransportAcc), st) != cudaSuccess) return SLG_ERR_CUDA;
  if (cudaMemsetAsync(&acc->ierr_key, 0xff, sizeof(unsigned long long), st) != cudaSuccess) return SLG_ERR_CUDA;
  if (cudaMemsetAsync(out->tally, 0, sizeof(double) * nx, st) != cudaSuccess) return SLG_ERR_CUDA;
  if (cudaMemsetAsync(out->jrad, 0, sizeof(double) * nx * ng, st) != cudaSuccess) return SLG_ERR_CUDA;
  if (cudaMemsetAsync(out->eamp, 0, sizeof(double) * nx, st) != cudaSuccess) return SLG_ERR_CUDA;
  if (in->dogrdtally && cudaMemsetAsync(out->methodswap, 0, sizeof(int32_t) * nx, st) != cudaSuccess)
    return SLG_ERR_CUDA;
  rc = launch_cell_tables_raw(st, (int)nx, (int)ng, nep, nepg, grid->xarr, grid->vxarr, grid->divv, grid->wlinv,
                              in, T);
  if (rc) return rc;
  TrnArgs A;
  A.nx = (int)nx; A.ng = (int)ng; A.nep = nep; A.nepg = nepg;
  A.xarr = grid->xarr; A.vxarr = grid->vxarr; A.divv = grid->divv; A.wl = grid->wl; A.wlinv = grid->wlinv;
  A.tempinv = in->tempinv; A.sig = in->sig; A.capgrey = in->capgrey; A.emitprob = in->emitprob;
  A.opaclump = in->opaclump; A.cap = in->cap; A.tauddmc = in->tauddmc; A.taulump = in->taulump;
  A.puretran = in->puretran; A.noampfact = in->noampfact; A.errorfatal = in->errorfatal;
  A.thm_aniso = in->thm_aniso; A.dogrdtally = in->dogrdtally; A.max_steps = in->max_steps;
  A.T = T; A.prt = prt; A.isvacant = isvacant; A.npart = npart; A.seed = seed;
  A.tally = out->tally; A.jrad = out->jrad; A.eamp = out->eamp; A.methodswap = out->methodswap;
  A.acc = acc; A.trace_hash = nullptr; A.trace_nstep = nullptr;
  int nsm = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return SLG_ERR_CUDA;
  long long nblk = (long long)nsm * particle_advance_blocks_per_sm();
  const long long need = (npart + particle_advance_block_size() - 1) / particle_advance_block_size();
  if (need < nblk) nblk = need > 0 ? need : 1;
  rc = launch_particle_advance_raw(st, A, (int)nblk);
  if (rc) return rc;
  TransportAcc h;
  if (cudaMemcpyAsync(&h, acc, sizeof(TransportAcc), cudaMemcpyDeviceToHost, st) != cudaSuccess) return SLG_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return SLG_ERR_CUDA;
  return finish_particle_advance_acc(h, out);
}
