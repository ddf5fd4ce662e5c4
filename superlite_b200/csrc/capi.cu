// capi.cu -- extern "C" entry points of libslg (declared in include/slg.h).
//
// Host-pointer entry points stage their arrays in context-owned device
// buffers, call the device-pointer form on the context's stream, copy the
// outputs back and synchronise.  Device-pointer entry points only queue work.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <algorithm>
#include "slg.h"
#include "slg_internal.h"

namespace slg {

int set_error(slg_ctx* ctx, int code, const char* fmt, ...) {
  if (!ctx) return code;
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  ctx->err = buf;
  if (ctx->capturing) ctx->capture_failed = 1;  // the graph would miss this call's work
  return code;
}

int cuda_check(slg_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SLG_OK;
  return set_error(ctx, SLG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

void* scratch(slg_ctx* ctx, int slot, size_t bytes) {
  DevBuf& b = ctx->scratch[slot];
  if (bytes == 0) bytes = 16;
  if (b.bytes >= bytes) return b.p;
  if (b.p) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    if ((slot >= 12 && slot <= 20) || slot == 72) ctx->tables.nx = ctx->tables.ng = 0;
  }
  const size_t alloc = bytes + bytes / 8;  // headroom for small growth
  if (cudaMalloc(&b.p, alloc) != cudaSuccess) {
    cudaGetLastError();
    set_error(ctx, SLG_ERR_OOM, "cudaMalloc of %zu bytes failed", alloc);
    return nullptr;
  }
  b.bytes = alloc;
  return b.p;
}

int opacity_flags(slg_ctx* ctx, int32_t* sanity, int32_t* binning);
int sourcetally_error(slg_ctx* ctx, int* err);
int finish_particle_advance_acc(const TransportAcc& a, slg_transport_out* out);
void host_sourceenergy(int nx, const double* xarr, const double* radtemp, double L_bol, double* emit,
                       double* tot_sthermal);
long long host_sourcenumbers(int nx, const double* emit, double pwr, long long src_ns, long long nvacant,
                             int32_t* nvol);
int launch_interior_source(slg_ctx* ctx, const double* d_radtemp, const double* h_emit, const int32_t* h_nvol,
                           long long npart, slg_packet* prt, int32_t* isvacant, uint64_t seed, long long* nnew_out);
int interior_source_check(slg_ctx* ctx, long long nnew);
int autotune_transport(slg_ctx* ctx, const slg_transport_in* in, const slg_packet* prt, const int32_t* isvacant,
                       int64_t npart, uint64_t seed, int64_t nsample, int* best, float* ms);

}  // namespace slg

using namespace slg;

namespace {

// Staging slots used by the host-pointer entry points.
enum {
  H_A = 32, H_B, H_C, H_D, H_E, H_F, H_G, H_H, H_I, H_J, H_K, H_L, H_M, H_N, H_O, H_P
};

template <class T>
T* up(slg_ctx* ctx, int slot, const T* h, size_t n, int* rc) {
  if (*rc) return nullptr;
  if (!h) return nullptr;
  T* d = (T*)scratch(ctx, slot, sizeof(T) * n);
  if (!d) { *rc = SLG_ERR_OOM; return nullptr; }
  *rc = cuda_check(ctx, cudaMemcpyAsync(d, h, sizeof(T) * n, cudaMemcpyHostToDevice, ctx->stream), "upload");
  return d;
}
template <class T>
T* out_buf(slg_ctx* ctx, int slot, size_t n, int* rc) {
  if (*rc) return nullptr;
  T* d = (T*)scratch(ctx, slot, sizeof(T) * n);
  if (!d) *rc = SLG_ERR_OOM;
  return d;
}
template <class T>
void down(slg_ctx* ctx, T* h, const T* d, size_t n, int* rc) {
  if (*rc || !h || !d) return;
  *rc = cuda_check(ctx, cudaMemcpyAsync(h, d, sizeof(T) * n, cudaMemcpyDeviceToHost, ctx->stream), "download");
}
int finish(slg_ctx* ctx, int rc) {
  const int rs = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "stream sync");
  return rc ? rc : rs;
}
bool need_grid(slg_ctx* ctx) { return ctx->nx > 0 && ctx->ng > 0; }

void free_dev(void* p) {
  if (p) cudaFree(p);
}

// The grid of one or more models (grid_setup per model, GRID/grid_setup.f:3-62):
// per-model shell edges one model after another, per-cell arrays over all cells.
int set_models(slg_ctx* ctx, const char* fn, int nmodel, const int32_t* nx, const int64_t* npart,
               const double* xarr, const double* vxarr, const double* vol, const double* divv) {
  if (!ctx || nmodel < 1 || !nx || !xarr || !vxarr || !vol || !divv)
    return set_error(ctx, SLG_ERR_ARG, "%s: bad arguments", fn);
  if (ctx->capturing) return set_error(ctx, SLG_ERR_STATE, "%s: a graph capture is open", fn);
  std::vector<ModelDesc> md(nmodel);
  long long nc = 0, np = 0;
  for (int m = 0; m < nmodel; ++m) {
    if (nx[m] < 1 || (nmodel > 1 && nx[m] < 2))
      return set_error(ctx, SLG_ERR_ARG, "%s: model %d has %d shells", fn, m, nx[m]);
    if (npart && npart[m] < 0) return set_error(ctx, SLG_ERR_ARG, "%s: model %d has %lld particles", fn, m,
                                                (long long)npart[m]);
    const double* X = xarr + nc + m;
    for (int k = 0; k < nx[m]; ++k)
      if (!(X[k + 1] > X[k]))
        return set_error(ctx, SLG_ERR_ARG, "%s: xarr of model %d not increasing at %d", fn, m, k);
    md[m].poff = np;
    md[m].np = npart ? npart[m] : 0;
    md[m].nx = nx[m];
    md[m].co = (int)nc;
    md[m].xo = (int)(nc + m);
    md[m].pad = 0;
    nc += nx[m];
    np += md[m].np;
    if (nc > (1 << 30)) return set_error(ctx, SLG_ERR_ARG, "%s: too many shells", fn);
  }
  const int ncell = (int)nc, nedge = (int)nc + nmodel;
  std::vector<int4> cmap;
  if (nmodel > 1) {
    cmap.resize(ncell);
    for (int m = 0; m < nmodel; ++m)
      for (int i = 0; i < nx[m]; ++i) cmap[md[m].co + i] = make_int4(i + 1, nx[m], md[m].co, m);
  }
  cudaSetDevice(ctx->device);
  int rc = SLG_OK;
  if (ncell != ctx->nx || nmodel != ctx->nmodel) {
    free_dev(ctx->d_xarr); free_dev(ctx->d_vxarr); free_dev(ctx->d_vol); free_dev(ctx->d_divv);
    free_dev(ctx->d_models); free_dev(ctx->d_cellmap);
    ctx->d_xarr = ctx->d_vxarr = ctx->d_vol = ctx->d_divv = nullptr;
    ctx->d_models = nullptr;
    ctx->d_cellmap = nullptr;
    ctx->nx = 0;
    ctx->nmodel = 0;
    rc = cuda_check(ctx, cudaMalloc(&ctx->d_xarr, sizeof(double) * nedge), "alloc xarr");
    if (!rc) rc = cuda_check(ctx, cudaMalloc(&ctx->d_vxarr, sizeof(double) * nedge), "alloc vxarr");
    if (!rc) rc = cuda_check(ctx, cudaMalloc(&ctx->d_vol, sizeof(double) * ncell), "alloc vol");
    if (!rc) rc = cuda_check(ctx, cudaMalloc(&ctx->d_divv, sizeof(double) * ncell), "alloc divv");
    if (!rc) rc = cuda_check(ctx, cudaMalloc(&ctx->d_models, sizeof(ModelDesc) * nmodel), "alloc models");
    if (!rc && nmodel > 1) rc = cuda_check(ctx, cudaMalloc(&ctx->d_cellmap, sizeof(int4) * ncell), "alloc cellmap");
    if (rc) return rc;
  }
  cudaStream_t st = ctx->stream;
  rc = cuda_check(ctx, cudaMemcpyAsync(ctx->d_xarr, xarr, sizeof(double) * nedge, cudaMemcpyHostToDevice, st), "xarr");
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(ctx->d_vxarr, vxarr, sizeof(double) * nedge, cudaMemcpyHostToDevice, st), "vxarr");
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(ctx->d_vol, vol, sizeof(double) * ncell, cudaMemcpyHostToDevice, st), "vol");
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(ctx->d_divv, divv, sizeof(double) * ncell, cudaMemcpyHostToDevice, st), "divv");
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(ctx->d_models, md.data(), sizeof(ModelDesc) * nmodel, cudaMemcpyHostToDevice, st), "models");
  if (!rc && nmodel > 1)
    rc = cuda_check(ctx, cudaMemcpyAsync(ctx->d_cellmap, cmap.data(), sizeof(int4) * ncell, cudaMemcpyHostToDevice, st), "cellmap");
  if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(st), "grid sync");
  if (rc) return rc;
  ctx->nx = ncell;
  ctx->nmodel = nmodel;
  ctx->h_models = md;
  ctx->npart_models = npart ? np : 0;
  ctx->h_xarr.assign(xarr, xarr + nedge);
  ctx->tables.nx = ctx->tables.ng = 0;
  ctx->src_emit.clear();
  ctx->src_nvol.clear();
  return SLG_OK;
}

// Zero the running transport counters (first error: none).
int reset_totals(slg_ctx* ctx) {
  int rc = cuda_check(ctx, cudaMemsetAsync(ctx->d_totals, 0, sizeof(TransportAcc), ctx->stream), "totals");
  if (!rc)
    rc = cuda_check(ctx, cudaMemsetAsync(&ctx->d_totals->ierr_key, 0xff, sizeof(unsigned long long), ctx->stream),
                    "totals");
  return rc;
}

__global__ void epoch_bump_kernel(unsigned long long* e) { *e += 1ull; }

int check_model_particles(slg_ctx* ctx, int64_t npart);

// fluxtally per model: model m's escaped particles go to rows m of
// luminos/lumdev/lumnum (flx_ng entries each).
int fluxtally_models(slg_ctx* ctx, int64_t npart, const slg_packet* prt, int32_t* isvacant, int flx_ng,
                     const double* flx_wl, double* luminos, double* lumdev, int32_t* lumnum) {
  if (ctx->nmodel <= 1) return launch_fluxtally(ctx, npart, prt, isvacant, flx_ng, flx_wl, luminos, lumdev, lumnum);
  int rc = check_model_particles(ctx, npart);
  for (int m = 0; m < ctx->nmodel && !rc; ++m) {
    const ModelDesc& d = ctx->h_models[m];
    const size_t o = (size_t)m * flx_ng;
    rc = launch_fluxtally(ctx, d.np, prt + d.poff, isvacant + d.poff, flx_ng, flx_wl, luminos + o, lumdev + o,
                          lumnum + o);
  }
  return rc;
}

// Particle count of a call against the models' slot ranges.
int check_model_particles(slg_ctx* ctx, int64_t npart) {
  if (ctx->nmodel > 1 && npart != ctx->npart_models)
    return set_error(ctx, SLG_ERR_ARG, "npart %lld differs from the %lld slots of the models", (long long)npart,
                     ctx->npart_models);
  return SLG_OK;
}

}  // namespace

extern "C" {

const char* slg_version(void) { return "superlite_b200 libslg sm_100a " __DATE__; }

slg_ctx* slg_create(int device) {
  if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return nullptr; }
  slg_ctx* ctx = new slg_ctx();
  ctx->device = device;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete ctx;
    return nullptr;
  }
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaMalloc(&ctx->d_acc, sizeof(TransportAcc)) != cudaSuccess ||
      cudaMallocHost(&ctx->h_acc, sizeof(TransportAcc)) != cudaSuccess ||
      cudaMalloc(&ctx->d_totals, sizeof(TransportAcc)) != cudaSuccess ||
      cudaMalloc(&ctx->d_epoch, sizeof(unsigned long long)) != cudaSuccess ||
      reset_totals(ctx) != SLG_OK || cudaMemset(ctx->d_epoch, 0, sizeof(unsigned long long)) != cudaSuccess ||
      cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
    cudaGetLastError();
    slg_destroy(ctx);
    return nullptr;
  }
  std::memset(ctx->h_acc, 0, sizeof(TransportAcc));
  return ctx;
}

void slg_destroy(slg_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& b : ctx->scratch) free_dev(b.p);
  free_dev(ctx->d_wl); free_dev(ctx->d_wlinv);
  free_dev(ctx->d_xarr); free_dev(ctx->d_vxarr); free_dev(ctx->d_vol); free_dev(ctx->d_divv);
  free_dev(ctx->d_ion_ni); free_dev(ctx->d_bb); free_dev(ctx->d_ph1); free_dev(ctx->d_ph2);
  free_dev(ctx->d_gff); free_dev(ctx->d_acc);
  free_dev(ctx->d_totals); free_dev(ctx->d_epoch); free_dev(ctx->d_models); free_dev(ctx->d_cellmap);
  free_dev(ctx->d_eos_ni); free_dev(ctx->d_eos_e); free_dev(ctx->d_eos_q); free_dev(ctx->d_eos_g1);
  free_dev(ctx->d_amass); free_dev(ctx->d_lrow_of_slot); free_dev(ctx->d_slot_of_lrow);
  if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
  if (ctx->h_acc) cudaFreeHost(ctx->h_acc);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* slg_last_error(const slg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void* slg_stream(slg_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int slg_sync(slg_ctx* ctx) {
  if (!ctx) return SLG_ERR_ARG;
  if (ctx->capturing) return set_error(ctx, SLG_ERR_STATE, "slg_sync: a graph capture is open");
  int rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "stream sync");
  if (!rc && ctx->pending_out) {
    slg_transport_out* o = ctx->pending_out;
    ctx->pending_out = nullptr;
    rc = finish_particle_advance(ctx, nullptr, o);
  }
  return rc;
}

// ------------------------------------------------------------------ CUDA graphs
int slg_graph_begin(slg_ctx* ctx) {
  if (!ctx) return SLG_ERR_ARG;
  if (ctx->capturing) return set_error(ctx, SLG_ERR_STATE, "slg_graph_begin: a capture is already open");
  int rc = slg_sync(ctx);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  rc = cuda_check(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
  if (!rc) {
    ctx->capturing = 1;
    ctx->capture_failed = 0;
  }
  return rc;
}

int slg_graph_end(slg_ctx* ctx) {
  if (!ctx) return SLG_ERR_ARG;
  if (!ctx->capturing) return set_error(ctx, SLG_ERR_STATE, "slg_graph_end: no capture is open");
  cudaSetDevice(ctx->device);
  epoch_bump_kernel<<<1, 1, 0, ctx->stream>>>(ctx->d_epoch);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  ctx->capturing = 0;
  ctx->pending_out = nullptr;  // captured calls complete on replay (slg_transport_totals)
  if (ctx->capture_failed && e == cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return set_error(ctx, SLG_ERR_STATE, "slg_graph_end: a call failed during the capture (%s)", ctx->err.c_str());
  }
  if (e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return set_error(ctx, SLG_ERR_CUDA, "slg_graph_end: capture failed (%s); a call during the capture needed "
                     "an allocation, an upload of changed host data or a host wait", cudaGetErrorString(e));
  }
  if (ctx->graph_exec) {
    cudaGraphExecDestroy(ctx->graph_exec);
    ctx->graph_exec = nullptr;
  }
  int rc = cuda_check(ctx, cudaGraphInstantiate(&ctx->graph_exec, g, 0), "graph instantiate");
  cudaGraphDestroy(g);
  if (!rc) rc = cuda_check(ctx, cudaMemsetAsync(ctx->d_epoch, 0, sizeof(unsigned long long), ctx->stream), "epoch");
  return rc;
}

int slg_graph_launch(slg_ctx* ctx, int32_t nlaunch) {
  if (!ctx || nlaunch < 0) return set_error(ctx, SLG_ERR_ARG, "slg_graph_launch: bad argument");
  if (!ctx->graph_exec || ctx->capturing) return set_error(ctx, SLG_ERR_STATE, "slg_graph_launch: no graph");
  cudaSetDevice(ctx->device);
  for (int i = 0; i < nlaunch; ++i) {
    const int rc = cuda_check(ctx, cudaGraphLaunch(ctx->graph_exec, ctx->stream), "graph launch");
    if (rc) return rc;
  }
  return SLG_OK;
}

int slg_transport_totals(slg_ctx* ctx, slg_transport_out* out, int32_t reset) {
  if (!ctx || !out) return set_error(ctx, SLG_ERR_ARG, "slg_transport_totals: bad argument");
  int rc = slg_sync(ctx);
  if (rc > 0) rc = SLG_OK;  // a transport error of the last direct call is reported below as well
  if (rc) return rc;
  TransportAcc h;
  rc = cuda_check(ctx, cudaMemcpy(&h, ctx->d_totals, sizeof(TransportAcc), cudaMemcpyDeviceToHost), "totals");
  if (rc) return rc;
  out->tot_evelo = out->tot_eout = out->tot_sflux = 0.0;
  const int ierr = finish_particle_advance_acc(h, out);
  if (reset) {
    rc = reset_totals(ctx);
    if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "totals reset");
    if (rc) return rc;
  }
  return ierr;
}

int slg_set_groups(slg_ctx* ctx, int32_t ng, const double* grp_wl) {
  if (!ctx || ng < 1 || !grp_wl) return set_error(ctx, SLG_ERR_ARG, "slg_set_groups: bad arguments");
  if (ng > SLG_MAX_GROUPS)
    return set_error(ctx, SLG_ERR_TOO_LARGE, "slg_set_groups: %d groups > SLG_MAX_GROUPS (%d)", ng, SLG_MAX_GROUPS);
  for (int k = 0; k < ng; ++k)
    if (!(grp_wl[k + 1] > grp_wl[k]) || !(grp_wl[k] > 0.0))
      return set_error(ctx, SLG_ERR_ARG, "slg_set_groups: wavelength grid not increasing at %d", k);
  cudaSetDevice(ctx->device);
  free_dev(ctx->d_wl);
  free_dev(ctx->d_wlinv);
  ctx->d_wl = ctx->d_wlinv = nullptr;
  std::vector<double> inv(ng + 1);
  for (int k = 0; k <= ng; ++k) inv[k] = 1.0 / grp_wl[k];  // groupmod.f:51
  int rc = cuda_check(ctx, cudaMalloc(&ctx->d_wl, sizeof(double) * (ng + 1)), "alloc wl");
  if (!rc) rc = cuda_check(ctx, cudaMalloc(&ctx->d_wlinv, sizeof(double) * (ng + 1)), "alloc wlinv");
  if (!rc) rc = cuda_check(ctx, cudaMemcpy(ctx->d_wl, grp_wl, sizeof(double) * (ng + 1), cudaMemcpyHostToDevice), "wl");
  if (!rc) rc = cuda_check(ctx, cudaMemcpy(ctx->d_wlinv, inv.data(), sizeof(double) * (ng + 1), cudaMemcpyHostToDevice), "wlinv");
  if (rc) return rc;
  ctx->ng = ng;
  ctx->h_wl.assign(grp_wl, grp_wl + ng + 1);
  ctx->nep = (int)lround(std::sqrt((double)ng));                 // gridmod.f:121
  ctx->nepg = (int)std::ceil(ng / (ctx->nep + 1.0));              // gridmod.f:122
  ctx->tables.nx = ctx->tables.ng = 0;
  return SLG_OK;
}

int slg_set_grid(slg_ctx* ctx, int32_t nx, const double* xarr, const double* vxarr, const double* vol,
                 const double* divv) {
  return set_models(ctx, "slg_set_grid", 1, &nx, nullptr, xarr, vxarr, vol, divv);
}

int slg_set_models(slg_ctx* ctx, int32_t nmodel, const int32_t* nx, const int64_t* npart, const double* xarr,
                   const double* vxarr, const double* vol, const double* divv) {
  if (!npart) return set_error(ctx, SLG_ERR_ARG, "slg_set_models: npart is null");
  return set_models(ctx, "slg_set_models", nmodel, nx, npart, xarr, vxarr, vol, divv);
}

int slg_set_atomic_data(slg_ctx* ctx, int32_t nelem, int32_t nstage, const int32_t* ion_ni, int64_t nline,
                        const slg_bbxs* bb_xs, const float* bf_ph1, const float* bf_ph2, const double* ff_gff) {
  if (!ctx || nelem < 1 || nelem > 30 || nstage < 1 || nstage > 64 || !ion_ni || nline < 0 || (nline > 0 && !bb_xs))
    return set_error(ctx, SLG_ERR_ARG, "slg_set_atomic_data: bad arguments");
  if (nline > 0x7fffffffLL) return set_error(ctx, SLG_ERR_ARG, "slg_set_atomic_data: too many lines");
  for (int64_t l = 0; l + 1 < nline; ++l)
    if (!(bb_xs[l].wl0 <= bb_xs[l + 1].wl0))
      return set_error(ctx, SLG_ERR_UNSORTED, "slg_set_atomic_data: lines not sorted by wl0 at %lld", (long long)l);
  for (int64_t l = 0; l < nline; ++l)
    if (bb_xs[l].iz < 1 || bb_xs[l].iz > nelem || bb_xs[l].ii < 1 || bb_xs[l].ii > nstage)
      return set_error(ctx, SLG_ERR_ARG, "slg_set_atomic_data: line %lld has ion (%d,%d) outside the tables",
                       (long long)l, bb_xs[l].iz, bb_xs[l].ii);
  cudaSetDevice(ctx->device);
  free_dev(ctx->d_ion_ni); free_dev(ctx->d_bb); free_dev(ctx->d_ph1); free_dev(ctx->d_ph2); free_dev(ctx->d_gff);
  ctx->d_ion_ni = nullptr; ctx->d_bb = nullptr; ctx->d_ph1 = ctx->d_ph2 = nullptr; ctx->d_gff = nullptr;
  int rc = cuda_check(ctx, cudaMalloc(&ctx->d_ion_ni, sizeof(int32_t) * nelem), "alloc ion_ni");
  if (!rc) rc = cuda_check(ctx, cudaMemcpy(ctx->d_ion_ni, ion_ni, sizeof(int32_t) * nelem, cudaMemcpyHostToDevice), "ion_ni");
  if (!rc && nline > 0) {
    rc = cuda_check(ctx, cudaMalloc(&ctx->d_bb, sizeof(slg_bbxs) * nline), "alloc bb");
    if (!rc) rc = cuda_check(ctx, cudaMemcpy(ctx->d_bb, bb_xs, sizeof(slg_bbxs) * nline, cudaMemcpyHostToDevice), "bb");
  }
  if (!rc && bf_ph1 && bf_ph2) {
    rc = cuda_check(ctx, cudaMalloc(&ctx->d_ph1, sizeof(float) * 6 * 7 * 30 * 30), "alloc ph1");
    if (!rc) rc = cuda_check(ctx, cudaMalloc(&ctx->d_ph2, sizeof(float) * 7 * 30 * 30), "alloc ph2");
    if (!rc) rc = cuda_check(ctx, cudaMemcpy(ctx->d_ph1, bf_ph1, sizeof(float) * 6 * 7 * 30 * 30, cudaMemcpyHostToDevice), "ph1");
    if (!rc) rc = cuda_check(ctx, cudaMemcpy(ctx->d_ph2, bf_ph2, sizeof(float) * 7 * 30 * 30, cudaMemcpyHostToDevice), "ph2");
  }
  if (!rc && ff_gff) {
    rc = cuda_check(ctx, cudaMalloc(&ctx->d_gff, sizeof(double) * 81 * 41), "alloc gff");
    if (!rc) rc = cuda_check(ctx, cudaMemcpy(ctx->d_gff, ff_gff, sizeof(double) * 81 * 41, cudaMemcpyHostToDevice), "gff");
  }
  // the population rows the lines reference (the opacity adjoint accumulates
  // d cap / d population for those rows only)
  const int nslot = nelem * nstage;
  std::vector<int16_t> row_of(nslot, (int16_t)-1), slot_of;
  // the largest lower-level energy: the opacity kernels skip the range check
  // of their exp for a shell with hc/kT * chimax <= 700 (infinite when a
  // value is negative or NaN: every term is then checked)
  double chimax = 0.0;
  for (int64_t l = 0; l < nline; ++l) {
    const double c = (double)bb_xs[l].chilw;
    chimax = (c >= 0.0 && chimax < INFINITY) ? (c > chimax ? c : chimax) : INFINITY;
  }
  for (int64_t l = 0; l < nline; ++l) {
    const int sl = (bb_xs[l].iz - 1) * nstage + (bb_xs[l].ii - 1);
    if (row_of[sl] < 0) {
      row_of[sl] = (int16_t)slot_of.size();
      slot_of.push_back((int16_t)sl);
    }
  }
  free_dev(ctx->d_lrow_of_slot); free_dev(ctx->d_slot_of_lrow);
  ctx->d_lrow_of_slot = ctx->d_slot_of_lrow = nullptr;
  if (!rc) rc = cuda_check(ctx, cudaMalloc(&ctx->d_lrow_of_slot, sizeof(int16_t) * nslot), "alloc row map");
  if (!rc) rc = cuda_check(ctx, cudaMemcpy(ctx->d_lrow_of_slot, row_of.data(), sizeof(int16_t) * nslot,
                                          cudaMemcpyHostToDevice), "row map");
  if (!rc && !slot_of.empty()) {
    rc = cuda_check(ctx, cudaMalloc(&ctx->d_slot_of_lrow, sizeof(int16_t) * slot_of.size()), "alloc slot map");
    if (!rc) rc = cuda_check(ctx, cudaMemcpy(ctx->d_slot_of_lrow, slot_of.data(), sizeof(int16_t) * slot_of.size(),
                                            cudaMemcpyHostToDevice), "slot map");
  }
  if (rc) return rc;
  ctx->nelem = nelem;
  ctx->nstage = nstage;
  ctx->nline = nline;
  ctx->nlrow = (int)slot_of.size();
  ctx->line_chimax = chimax;
  ctx->h_ion_ni.assign(ion_ni, ion_ni + nelem);
  return SLG_OK;
}

int slg_set_trace(slg_ctx* ctx, uint64_t* trace_hash, int32_t* trace_nstep) {
  if (!ctx) return SLG_ERR_ARG;
  ctx->trace_hash = trace_hash;
  ctx->trace_nstep = trace_nstep;
  return SLG_OK;
}

// ------------------------------------------------------------------ device forms
int slg_dev_physical_opacity(slg_ctx* ctx, const slg_gas* gas, const slg_opacity_flags* flags, double* gas_sig,
                             float* gas_cap, float* gas_emiss, double* cap64) {
  if (!ctx || !gas || !flags || !gas_sig || !gas_cap || !gas_emiss) return set_error(ctx, SLG_ERR_ARG, "null argument");
  if (!need_grid(ctx)) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  cudaSetDevice(ctx->device);
  return launch_physical_opacity(ctx, gas, flags, gas_sig, gas_cap, gas_emiss, cap64);
}

int slg_dev_opacity_means(slg_ctx* ctx, const double* temp, const double* sig, const float* gas_cap, double* capgrey,
                          double* capross) {
  if (!ctx || !temp || !gas_cap || !capgrey) return set_error(ctx, SLG_ERR_ARG, "null argument");
  if (!need_grid(ctx)) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  cudaSetDevice(ctx->device);
  return launch_opacity_means(ctx, temp, sig, gas_cap, capgrey, capross);
}

int slg_dev_leakage_opacity11(slg_ctx* ctx, const double* tempinv, const double* sig, const float* cap,
                              const float* capemit, double tauddmc, double taulump, double* opaclump) {
  if (!ctx || !tempinv || !sig || !cap || !opaclump) return set_error(ctx, SLG_ERR_ARG, "null argument");
  if (!need_grid(ctx)) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  cudaSetDevice(ctx->device);
  return launch_leakage(ctx, tempinv, sig, cap, capemit, tauddmc, taulump, opaclump);
}

int slg_dev_emission_probability(slg_ctx* ctx, const double* tempinv, const float* cap, const double* capgrey,
                                 double* emitprob) {
  if (!ctx || !tempinv || !cap || !capgrey || !emitprob) return set_error(ctx, SLG_ERR_ARG, "null argument");
  if (!need_grid(ctx)) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  cudaSetDevice(ctx->device);
  return launch_emitprob(ctx, tempinv, cap, capgrey, emitprob);
}

int slg_dev_particle_advance(slg_ctx* ctx, const slg_transport_in* in, slg_packet* prt, int32_t* isvacant,
                             int64_t npart, uint64_t seed, slg_transport_out* out) {
  if (!ctx || !in || !out || (npart > 0 && (!prt || !isvacant)) || npart < 0)
    return set_error(ctx, SLG_ERR_ARG, "null argument");
  if (!in->tempinv || !in->sig || !in->capgrey || !in->emitprob || !in->opaclump || !in->cap)
    return set_error(ctx, SLG_ERR_ARG, "slg_transport_in has a null array");
  if (!out->tally || !out->jrad || !out->eamp || (in->dogrdtally && !out->methodswap))
    return set_error(ctx, SLG_ERR_ARG, "slg_transport_out has a null array");
  if (!need_grid(ctx)) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  if (ctx->nx < 2) return set_error(ctx, SLG_ERR_ARG, "transport needs at least 2 shells");
  if (in->precision != 0 && in->precision != 1)
    return set_error(ctx, SLG_ERR_NOT_BUILT, "precision %d not available", in->precision);
  if (check_model_particles(ctx, npart)) return SLG_ERR_ARG;
  cudaSetDevice(ctx->device);
  const int rc = launch_particle_advance(ctx, in, prt, isvacant, npart, seed, out, nullptr, nullptr);
  ctx->pending_out = rc ? nullptr : out;
  return rc;
}

int slg_dev_fluxtally(slg_ctx* ctx, int64_t npart, const slg_packet* prt, int32_t* isvacant, int32_t flx_ng,
                      const double* flx_wl, double* luminos, double* lumdev, int32_t* lumnum) {
  if (!ctx || flx_ng < 1 || !flx_wl || !luminos || !lumdev || !lumnum || npart < 0)
    return set_error(ctx, SLG_ERR_ARG, "bad argument");
  cudaSetDevice(ctx->device);
  return fluxtally_models(ctx, npart, prt, isvacant, flx_ng, flx_wl, luminos, lumdev, lumnum);
}

int slg_dev_sourcetally(slg_ctx* ctx, int64_t npart, const slg_packet* prt, const int32_t* isvacant,
                        double* src_energy, int32_t* src_number) {
  if (!ctx || !src_energy || !src_number || npart < 0) return set_error(ctx, SLG_ERR_ARG, "bad argument");
  if (!need_grid(ctx)) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  cudaSetDevice(ctx->device);
  return launch_sourcetally(ctx, npart, prt, isvacant, src_energy, src_number);
}

// ------------------------------------------------------------------ host forms
int slg_physical_opacity(slg_ctx* ctx, const slg_gas* gas, const slg_opacity_flags* flags, double* gas_sig,
                         float* gas_cap, float* gas_emiss, double* cap64, int32_t* sanity) {
  if (!ctx || !gas || !flags || !gas_sig || !gas_cap || !gas_emiss) return set_error(ctx, SLG_ERR_ARG, "null argument");
  if (!need_grid(ctx) || ctx->nelem < 1) return set_error(ctx, SLG_ERR_STATE, "groups/grid/atomic data not set");
  cudaSetDevice(ctx->device);
  const size_t nc = ctx->nx, ng = ctx->ng, ns = (size_t)ctx->nstage * ctx->nelem;
  int rc = 0;
  slg_gas d;
  d.temp = up(ctx, H_A, gas->temp, nc, &rc);
  d.natom = up(ctx, H_B, gas->natom, nc, &rc);
  d.nelec = up(ctx, H_C, gas->nelec, nc, &rc);
  d.vol = up(ctx, H_D, gas->vol, nc, &rc);
  d.mass = up(ctx, H_E, gas->mass, nc, &rc);
  d.natomfr = up(ctx, H_F, gas->natomfr, nc * (ctx->nelem + 1), &rc);
  d.oc = up(ctx, H_G, gas->oc, nc * ns, &rc);
  d.ginv = up(ctx, H_H, gas->ginv, nc * ns, &rc);
  double* dsig = out_buf<double>(ctx, H_I, nc, &rc);
  float* dcap = out_buf<float>(ctx, H_J, nc * ng, &rc);
  float* dem = out_buf<float>(ctx, H_K, nc * ng, &rc);
  double* dc64 = cap64 ? out_buf<double>(ctx, H_L, nc * ng, &rc) : nullptr;
  if (!rc && (!d.temp || !d.natom || !d.nelec || !d.vol || !d.mass || !d.natomfr || !d.oc || !d.ginv))
    rc = set_error(ctx, SLG_ERR_ARG, "slg_gas has a null array");
  if (!rc) rc = launch_physical_opacity(ctx, &d, flags, dsig, dcap, dem, dc64);
  down(ctx, gas_sig, dsig, nc, &rc);
  down(ctx, gas_cap, dcap, nc * ng, &rc);
  down(ctx, gas_emiss, dem, nc * ng, &rc);
  if (cap64) down(ctx, cap64, dc64, nc * ng, &rc);
  rc = finish(ctx, rc);
  if (!rc) {
    int32_t s = 0, b = 0;
    rc = opacity_flags(ctx, &s, &b);
    if (!rc && (b & 1)) rc = set_error(ctx, SLG_ERR_UNSORTED, "bb line list not sorted by wl0");
    if (!rc && (b & 2)) rc = set_error(ctx, SLG_ERR_CUDA, "line binning: shared-memory staging timed out");
    if (sanity) *sanity = s;
  }
  return rc;
}

int slg_analytic_opacity(slg_ctx* ctx, const double* temp, const double* rho, int32_t kind, double capcoef,
                         double captpwr, double caprpwr, double sigcoef, double sigtpwr, double sigrpwr,
                         double ldisp1, double ldisp2, double* gas_sig, float* gas_cap) {
  if (!ctx || !temp || !rho || !gas_sig || !gas_cap || kind < 1 || kind > 3)
    return set_error(ctx, SLG_ERR_ARG, "bad argument");
  if (!need_grid(ctx)) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  cudaSetDevice(ctx->device);
  const size_t nc = ctx->nx, ng = ctx->ng;
  int rc = 0;
  const double* dt = up(ctx, H_A, temp, nc, &rc);
  const double* dr = up(ctx, H_B, rho, nc, &rc);
  double* ds = out_buf<double>(ctx, H_I, nc, &rc);
  float* dc = out_buf<float>(ctx, H_J, nc * ng, &rc);
  const double c[8] = {capcoef, captpwr, caprpwr, sigcoef, sigtpwr, sigrpwr, ldisp1, ldisp2};
  if (!rc) rc = launch_analytic_opacity(ctx, dt, dr, kind, c, ds, dc);
  down(ctx, gas_sig, ds, nc, &rc);
  down(ctx, gas_cap, dc, nc * ng, &rc);
  return finish(ctx, rc);
}

int slg_dev_analytic_opacity(slg_ctx* ctx, const double* temp, const double* rho, int32_t kind, double capcoef,
                             double captpwr, double caprpwr, double sigcoef, double sigtpwr, double sigrpwr,
                             double ldisp1, double ldisp2, double* gas_sig, float* gas_cap) {
  if (!ctx || !temp || !rho || !gas_sig || !gas_cap || kind < 1 || kind > 3)
    return set_error(ctx, SLG_ERR_ARG, "bad argument");
  if (!need_grid(ctx)) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  cudaSetDevice(ctx->device);
  const double c[8] = {capcoef, captpwr, caprpwr, sigcoef, sigtpwr, sigrpwr, ldisp1, ldisp2};
  return launch_analytic_opacity(ctx, temp, rho, kind, c, gas_sig, gas_cap);
}

int slg_opacity_means(slg_ctx* ctx, const double* temp, const double* sig, const float* gas_cap, double* capgrey,
                      double* capross) {
  if (!ctx || !temp || !gas_cap || !capgrey) return set_error(ctx, SLG_ERR_ARG, "null argument");
  if (!need_grid(ctx)) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  cudaSetDevice(ctx->device);
  const size_t nc = ctx->nx, ng = ctx->ng;
  int rc = 0;
  const double* dt = up(ctx, H_A, temp, nc, &rc);
  const double* ds = up(ctx, H_B, sig, nc, &rc);
  const float* dc = up(ctx, H_C, gas_cap, nc * ng, &rc);
  double* dg = out_buf<double>(ctx, H_I, nc, &rc);
  double* dr = capross ? out_buf<double>(ctx, H_K, nc, &rc) : nullptr;
  if (!rc) rc = launch_opacity_means(ctx, dt, ds, dc, dg, dr);
  down(ctx, capgrey, dg, nc, &rc);
  if (capross) down(ctx, capross, dr, nc, &rc);
  return finish(ctx, rc);
}

int slg_leakage_opacity11(slg_ctx* ctx, const double* tempinv, const double* sig, const float* cap,
                          const float* capemit, double tauddmc, double taulump, double* opaclump) {
  if (!ctx || !tempinv || !sig || !cap || !opaclump) return set_error(ctx, SLG_ERR_ARG, "null argument");
  if (!need_grid(ctx)) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  cudaSetDevice(ctx->device);
  const size_t nc = ctx->nx, ng = ctx->ng;
  int rc = 0;
  const double* dt = up(ctx, H_A, tempinv, nc, &rc);
  const double* ds = up(ctx, H_B, sig, nc, &rc);
  const float* dc = up(ctx, H_C, cap, nc * ng, &rc);
  const float* de = capemit ? up(ctx, H_D, capemit, nc * ng, &rc) : nullptr;
  double* dol = out_buf<double>(ctx, H_I, nc * 11, &rc);
  if (!rc) rc = launch_leakage(ctx, dt, ds, dc, de, tauddmc, taulump, dol);
  down(ctx, opaclump, dol, nc * 11, &rc);
  return finish(ctx, rc);
}

int slg_emission_probability(slg_ctx* ctx, const double* tempinv, const float* cap, const double* capgrey,
                             double* emitprob) {
  if (!ctx || !tempinv || !cap || !capgrey || !emitprob) return set_error(ctx, SLG_ERR_ARG, "null argument");
  if (!need_grid(ctx)) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  cudaSetDevice(ctx->device);
  const size_t nc = ctx->nx, ng = ctx->ng;
  int rc = 0;
  const double* dt = up(ctx, H_A, tempinv, nc, &rc);
  const float* dc = up(ctx, H_C, cap, nc * ng, &rc);
  const double* dg = up(ctx, H_B, capgrey, nc, &rc);
  double* dep = out_buf<double>(ctx, H_I, nc * ctx->nep, &rc);
  if (!rc) rc = launch_emitprob(ctx, dt, dc, dg, dep);
  down(ctx, emitprob, dep, nc * ctx->nep, &rc);
  return finish(ctx, rc);
}

int slg_particle_advance(slg_ctx* ctx, const slg_transport_in* in, slg_packet* prt, int32_t* isvacant, int64_t npart,
                         uint64_t seed, slg_transport_out* out) {
  if (!ctx || !in || !out || (npart > 0 && (!prt || !isvacant)) || npart < 0)
    return set_error(ctx, SLG_ERR_ARG, "null argument");
  if (!in->tempinv || !in->sig || !in->capgrey || !in->emitprob || !in->opaclump || !in->cap)
    return set_error(ctx, SLG_ERR_ARG, "slg_transport_in has a null array");
  if (!out->tally || !out->jrad || !out->eamp || (in->dogrdtally && !out->methodswap))
    return set_error(ctx, SLG_ERR_ARG, "slg_transport_out has a null array");
  if (!need_grid(ctx)) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  if (ctx->nx < 2) return set_error(ctx, SLG_ERR_ARG, "transport needs at least 2 shells");
  if (in->precision != 0 && in->precision != 1)
    return set_error(ctx, SLG_ERR_NOT_BUILT, "precision %d not available", in->precision);
  if (check_model_particles(ctx, npart)) return SLG_ERR_ARG;
  cudaSetDevice(ctx->device);
  const size_t nc = ctx->nx, ng = ctx->ng, np = (size_t)npart;
  int rc = 0;
  slg_transport_in d = *in;
  d.tempinv = up(ctx, H_A, in->tempinv, nc, &rc);
  d.sig = up(ctx, H_B, in->sig, nc, &rc);
  d.capgrey = up(ctx, H_C, in->capgrey, nc, &rc);
  d.emitprob = up(ctx, H_D, in->emitprob, nc * ctx->nep, &rc);
  d.opaclump = up(ctx, H_E, in->opaclump, nc * 11, &rc);
  d.cap = up(ctx, H_F, in->cap, nc * ng, &rc);
  slg_packet* dp = up(ctx, H_G, prt, np, &rc);
  int32_t* dv = up(ctx, H_H, isvacant, np, &rc);
  slg_transport_out o = *out;
  o.tally = out_buf<double>(ctx, H_I, nc, &rc);
  o.jrad = out_buf<double>(ctx, H_J, nc * ng, &rc);
  o.eamp = out_buf<double>(ctx, H_K, nc, &rc);
  o.methodswap = out_buf<int32_t>(ctx, H_L, nc, &rc);
  if (ctx->nmodel > 1 && (ctx->trace_hash || ctx->trace_nstep))
    return set_error(ctx, SLG_ERR_ARG, "per-particle traces are for one-model contexts");
  uint64_t* dth = ctx->trace_hash ? out_buf<uint64_t>(ctx, H_M, np, &rc) : nullptr;
  int32_t* dtn = ctx->trace_nstep ? out_buf<int32_t>(ctx, H_N, np, &rc) : nullptr;
  if (!rc && dth) cudaMemsetAsync(dth, 0, sizeof(uint64_t) * np, ctx->stream);
  if (!rc && dtn) cudaMemsetAsync(dtn, 0, sizeof(int32_t) * np, ctx->stream);
  if (!rc) rc = launch_particle_advance(ctx, &d, dp, dv, npart, seed, &o, dth, dtn);
  down(ctx, prt, dp, np, &rc);
  down(ctx, isvacant, dv, np, &rc);
  down(ctx, out->tally, o.tally, nc, &rc);
  down(ctx, out->jrad, o.jrad, nc * ng, &rc);
  down(ctx, out->eamp, o.eamp, nc, &rc);
  if (in->dogrdtally && out->methodswap) down(ctx, out->methodswap, o.methodswap, nc, &rc);
  if (dth) down(ctx, ctx->trace_hash, dth, np, &rc);
  if (dtn) down(ctx, ctx->trace_nstep, dtn, np, &rc);
  rc = finish(ctx, rc);
  if (rc) return rc;
  return finish_particle_advance(ctx, in, out);
}

int slg_fluxtally(slg_ctx* ctx, int64_t npart, const slg_packet* prt, int32_t* isvacant, int32_t flx_ng,
                  const double* flx_wl, double* luminos, double* lumdev, int32_t* lumnum) {
  if (!ctx || flx_ng < 1 || !flx_wl || !luminos || !lumdev || !lumnum || npart < 0 || (npart > 0 && (!prt || !isvacant)))
    return set_error(ctx, SLG_ERR_ARG, "bad argument");
  cudaSetDevice(ctx->device);
  const size_t np = (size_t)npart;
  int rc = 0;
  const size_t nf = (size_t)flx_ng * (ctx->nmodel > 1 ? ctx->nmodel : 1);  // per model
  const slg_packet* dp = up(ctx, H_G, prt, np, &rc);
  int32_t* dv = up(ctx, H_H, isvacant, np, &rc);
  const double* dw = up(ctx, H_A, flx_wl, (size_t)flx_ng + 1, &rc);
  double* dl = out_buf<double>(ctx, H_I, nf, &rc);
  double* dd = out_buf<double>(ctx, H_J, nf, &rc);
  int32_t* dn = out_buf<int32_t>(ctx, H_K, nf, &rc);
  if (!rc) rc = fluxtally_models(ctx, npart, dp, dv, flx_ng, dw, dl, dd, dn);
  down(ctx, isvacant, dv, np, &rc);
  down(ctx, luminos, dl, nf, &rc);
  down(ctx, lumdev, dd, nf, &rc);
  down(ctx, lumnum, dn, nf, &rc);
  return finish(ctx, rc);
}

int slg_sourcetally(slg_ctx* ctx, int64_t npart, const slg_packet* prt, const int32_t* isvacant, double* src_energy,
                    int32_t* src_number) {
  if (!ctx || !src_energy || !src_number || npart < 0 || (npart > 0 && (!prt || !isvacant)))
    return set_error(ctx, SLG_ERR_ARG, "bad argument");
  if (!need_grid(ctx)) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  cudaSetDevice(ctx->device);
  const size_t np = (size_t)npart, n = (size_t)ctx->nx * ctx->ng;
  int rc = 0;
  const slg_packet* dp = up(ctx, H_G, prt, np, &rc);
  const int32_t* dv = up(ctx, H_H, isvacant, np, &rc);
  double* de = out_buf<double>(ctx, H_I, n, &rc);
  int32_t* dn = out_buf<int32_t>(ctx, H_J, n, &rc);
  if (!rc) rc = launch_sourcetally(ctx, npart, dp, dv, de, dn);
  down(ctx, src_energy, de, n, &rc);
  down(ctx, src_number, dn, n, &rc);
  rc = finish(ctx, rc);
  if (!rc) {
    int e = 0;
    rc = sourcetally_error(ctx, &e);
    if (!rc && (e & 1)) rc = set_error(ctx, SLG_ERR_ARG, "sourcetally: ic outside range");
    if (!rc && (e & 2)) rc = set_error(ctx, SLG_ERR_ARG, "sourcetally: ig outside range");
  }
  return rc;
}

// ------------------------------------------------------------------ autotuning
int slg_autotune_transport(slg_ctx* ctx, const slg_transport_in* in, const slg_packet* prt, const int32_t* isvacant,
                           int64_t npart, uint64_t seed, int64_t nsample, int32_t* best, float* ms) {
  if (!ctx || !in || npart < 0 || (npart > 0 && (!prt || !isvacant))) return set_error(ctx, SLG_ERR_ARG, "bad argument");
  if (!in->tempinv || !in->sig || !in->capgrey || !in->emitprob || !in->opaclump || !in->cap)
    return set_error(ctx, SLG_ERR_ARG, "slg_transport_in has a null array");
  if (!need_grid(ctx) || ctx->nx < 2) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  if (in->precision != 0 && in->precision != 1)
    return set_error(ctx, SLG_ERR_NOT_BUILT, "precision %d not available", in->precision);
  cudaSetDevice(ctx->device);
  int b = 0;
  const int rc = autotune_transport(ctx, in, prt, isvacant, npart, seed, nsample, &b, ms);
  if (best) *best = b;
  return rc;
}

int slg_set_transport_variant(slg_ctx* ctx, int32_t variant) {
  if (!ctx || variant < 0 || variant > 3) return set_error(ctx, SLG_ERR_ARG, "variant must be 0..3");
  ctx->trn_variant = variant;  // FP64 loop
  ctx->mix_variant = variant;  // mixed-precision loop
  return SLG_OK;
}

// ------------------------------------------------------------------ sources
int slg_sourceenergy(slg_ctx* ctx, const double* radtemp, double L_bol, double* emit, double* tot_sthermal) {
  if (!ctx || !radtemp || !emit) return set_error(ctx, SLG_ERR_ARG, "null argument");
  if (ctx->nx < 1) return set_error(ctx, SLG_ERR_STATE, "grid not set");
  double tot = 0.0;
  for (const ModelDesc& d : ctx->h_models) {  // each model renormalised to L_bol
    double t = 0.0;
    host_sourceenergy(d.nx, ctx->h_xarr.data() + d.xo, radtemp + d.co, L_bol, emit + d.co, &t);
    tot += t;
  }
  if (tot_sthermal) *tot_sthermal = tot;
  return SLG_OK;
}

int64_t slg_models_sourcenumbers(slg_ctx* ctx, const double* emit, double srcepwr, const int64_t* src_ns,
                                 const int64_t* nvacant, int32_t* nvol) {
  if (!ctx || !emit || !nvol || !src_ns || !nvacant) return set_error(ctx, SLG_ERR_ARG, "bad argument");
  if (ctx->nx < 1) return set_error(ctx, SLG_ERR_STATE, "grid not set");
  long long tot = 0;
  for (int m = 0; m < ctx->nmodel; ++m) {
    const ModelDesc& d = ctx->h_models[m];
    if (src_ns[m] < 1) return set_error(ctx, SLG_ERR_ARG, "model %d: src_ns %lld", m, (long long)src_ns[m]);
    const long long r = host_sourcenumbers(d.nx, emit + d.co, srcepwr, src_ns[m], nvacant[m], nvol + d.co);
    if (r < 0) return set_error(ctx, SLG_ERR_ARG, "sourcenumbers failed for model %d (%lld)", m, r);
    tot += r;
  }
  return tot;
}

int64_t slg_sourcenumbers(slg_ctx* ctx, const double* emit, double srcepwr, int64_t src_ns, int64_t nvacant,
                          int32_t* nvol) {
  if (!ctx || !emit || !nvol || src_ns < 1) return set_error(ctx, SLG_ERR_ARG, "bad argument");
  if (ctx->nx < 1) return set_error(ctx, SLG_ERR_STATE, "grid not set");
  if (ctx->nmodel > 1) return set_error(ctx, SLG_ERR_STATE, "several models: use slg_models_sourcenumbers");
  const long long r = host_sourcenumbers(ctx->nx, emit, srcepwr, src_ns, nvacant, nvol);
  if (r < 0) return set_error(ctx, SLG_ERR_ARG, "sourcenumbers failed (%lld)", r);
  return r;
}

int slg_dev_interior_source(slg_ctx* ctx, const double* radtemp, const double* emit, const int32_t* nvol,
                            slg_packet* prt, int32_t* isvacant, int64_t npart, uint64_t seed, int64_t* nnew) {
  if (!ctx || !radtemp || !emit || !nvol || npart < 0 || (npart > 0 && (!prt || !isvacant)))
    return set_error(ctx, SLG_ERR_ARG, "bad argument");
  if (!need_grid(ctx)) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  cudaSetDevice(ctx->device);
  long long n = 0;
  const int rc = launch_interior_source(ctx, radtemp, emit, nvol, npart, prt, isvacant, seed, &n);
  if (nnew) *nnew = n;
  return rc;
}

int slg_interior_source(slg_ctx* ctx, const double* radtemp, const double* emit, const int32_t* nvol,
                        slg_packet* prt, int32_t* isvacant, int64_t npart, uint64_t seed, int64_t* nnew) {
  if (!ctx || !radtemp || !emit || !nvol || npart < 0 || (npart > 0 && (!prt || !isvacant)))
    return set_error(ctx, SLG_ERR_ARG, "bad argument");
  if (!need_grid(ctx)) return set_error(ctx, SLG_ERR_STATE, "groups/grid not set");
  cudaSetDevice(ctx->device);
  const size_t np = (size_t)npart;
  int rc = 0;
  const double* dt = up(ctx, H_A, radtemp, (size_t)ctx->nx, &rc);
  slg_packet* dp = up(ctx, H_G, prt, np, &rc);
  int32_t* dv = up(ctx, H_H, isvacant, np, &rc);
  long long n = 0;
  if (!rc) rc = launch_interior_source(ctx, dt, emit, nvol, npart, dp, dv, seed, &n);
  down(ctx, prt, dp, np, &rc);
  down(ctx, isvacant, dv, np, &rc);
  rc = finish(ctx, rc);
  if (!rc) rc = interior_source_check(ctx, n);
  if (nnew) *nnew = n;
  return rc;
}

}  // extern "C"
