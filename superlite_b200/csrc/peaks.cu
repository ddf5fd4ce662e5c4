// peaks.cu -- throughput microbenchmarks of the pipes that bound the hot path
// (no counterpart in the reference): FP64 fused multiply-add, FP64 exp (the
// same device exp the opacity kernels evaluate once per line-shell term),
// FP32 fused multiply-add (one warp instruction per cycle per scheduler: the
// instruction-issue rate) and 32-bit integer multiply-add.
//
// Each thread runs CHAINS independent dependency chains (enough independent
// work to keep the pipe full) for `iters` rounds on a grid of 8 blocks of 256
// threads per SM, and writes one value so that the work cannot be removed.
// The host entry point times one launch with CUDA events on a private stream.
//
// slg_exp_eval evaluates the opacity kernels' table-driven FP64 exp
// (exp_tang, slg_device.cuh) on given arguments, for accuracy tests.
#include <cuda_runtime.h>
#include <cstdint>
#include "slg.h"
#include "slg_device.cuh"

namespace {

constexpr int PK_BLOCK = 256;
constexpr int PK_BLOCKS_PER_SM = 8;
constexpr int PK_CHAINS = 8;

__global__ void __launch_bounds__(PK_BLOCK) dfma_kernel(int iters, double a, double b, double* out) {
  double x[PK_CHAINS];
#pragma unroll
  for (int j = 0; j < PK_CHAINS; ++j) x[j] = 1e-3 * (threadIdx.x + 1) + j;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < PK_CHAINS; ++j) x[j] = fma(x[j], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < PK_CHAINS; ++j) s += x[j];
  out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// x <- exp(-x) keeps every chain in [exp(-1), 1]
__global__ void __launch_bounds__(PK_BLOCK) dexp_kernel(int iters, double* out) {
  double x[PK_CHAINS];
#pragma unroll
  for (int j = 0; j < PK_CHAINS; ++j) x[j] = 1e-4 * (threadIdx.x + 1) + 0.1 * j;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < PK_CHAINS; ++j) x[j] = exp(-x[j]);
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < PK_CHAINS; ++j) s += x[j];
  out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(PK_BLOCK) ffma_kernel(int iters, float a, float b, double* out) {
  float x[2 * PK_CHAINS];
#pragma unroll
  for (int j = 0; j < 2 * PK_CHAINS; ++j) x[j] = 1e-3f * (threadIdx.x + 1) + j;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 2 * PK_CHAINS; ++j) x[j] = fmaf(x[j], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < 2 * PK_CHAINS; ++j) s += x[j];
  out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(PK_BLOCK) imad_kernel(int iters, uint32_t a, uint32_t b, double* out) {
  uint32_t x[2 * PK_CHAINS];
#pragma unroll
  for (int j = 0; j < 2 * PK_CHAINS; ++j) x[j] = threadIdx.x * 2654435761u + j;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 2 * PK_CHAINS; ++j) x[j] = x[j] * a + b;
  }
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < 2 * PK_CHAINS; ++j) s ^= x[j];
  out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = (double)s;
}

__global__ void exp_eval_kernel(int64_t n, const double* __restrict__ x, double* __restrict__ y) {
  __shared__ double tab[slg::kExpTabN];
  slg::exp_table_load(tab);
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = slg::exp_tang(x[i], tab);
}

}  // namespace

namespace {
// The calling thread's current device, selected for the call and put back.
struct DeviceScope {
  int prev = -1;
  bool ok = false;
  explicit DeviceScope(int device) {
    ok = cudaGetDevice(&prev) == cudaSuccess && cudaSetDevice(device) == cudaSuccess;
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};
}  // namespace

extern "C" int slg_exp_eval(int device, int64_t n, const double* x, double* y) {
  if (n < 0 || (n > 0 && (!x || !y))) return SLG_ERR_ARG;
  if (n == 0) return SLG_OK;
  DeviceScope dev(device);
  if (!dev.ok) return SLG_ERR_CUDA;
  double* d = nullptr;
  if (cudaMalloc(&d, sizeof(double) * 2 * (size_t)n) != cudaSuccess) return SLG_ERR_OOM;
  int rc = SLG_OK;
  if (cudaMemcpy(d, x, sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess) rc = SLG_ERR_CUDA;
  if (!rc) {
    const int64_t nb = (n + 255) / 256;
    exp_eval_kernel<<<(unsigned)(nb < 4096 ? nb : 4096), 256>>>(n, d, d + n);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpy(y, d + n, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = SLG_ERR_CUDA;
  }
  cudaFree(d);
  return rc;
}

extern "C" int slg_pipe_throughput(int device, int which, int iters, double* ops_per_s, float* ms) {
  if (!ops_per_s || iters < 1 || which < 0 || which > 3) return SLG_ERR_ARG;
  DeviceScope dev(device);
  if (!dev.ok) return SLG_ERR_CUDA;
  int nsm = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return SLG_ERR_CUDA;
  const int nblk = nsm * PK_BLOCKS_PER_SM;
  const size_t nthr = (size_t)nblk * PK_BLOCK;
  double* out = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = SLG_OK;
  if (cudaMalloc(&out, sizeof(double) * nthr) != cudaSuccess) return SLG_ERR_OOM;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess)
    rc = SLG_ERR_CUDA;
  // operations counted per chain round: FMA = 2 flops, exp = 1 evaluation, IMAD = 1 operation
  double per_round = 0.0;
  for (int rep = 0; rep < 2 && !rc; ++rep) {  // the first launch warms up
    cudaEventRecord(e0, st);
    switch (which) {
      case 0: dfma_kernel<<<nblk, PK_BLOCK, 0, st>>>(iters, 0.999999, 1e-7, out); per_round = 2.0 * PK_CHAINS; break;
      case 1: dexp_kernel<<<nblk, PK_BLOCK, 0, st>>>(iters, out); per_round = PK_CHAINS; break;
      case 2: ffma_kernel<<<nblk, PK_BLOCK, 0, st>>>(iters, 0.9999f, 1e-6f, out); per_round = 4.0 * PK_CHAINS; break;
      default: imad_kernel<<<nblk, PK_BLOCK, 0, st>>>(iters, 1664525u, 1013904223u, out); per_round = 2.0 * PK_CHAINS;
    }
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = SLG_ERR_CUDA;
  }
  float t = 0.f;
  if (!rc && cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) rc = SLG_ERR_CUDA;
  if (!rc) {
    *ops_per_s = per_round * (double)iters * (double)nthr / (t * 1e-3);
    if (ms) *ms = t;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  cudaFree(out);
  return rc;
}
