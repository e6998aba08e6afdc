// tg_noalloc.cu -- residual norms for callers that cannot allocate device memory.
//
// tg_residual_norm_noalloc computes what compute_residual_norm computes
// (src/fv.cc:1801-1879) from caller-owned device buffers, without a handle and
// without allocating anything: its per-block partial sums live in the
// fixed-size device array below.  It exists for callers that must not call
// cudaMalloc once they are running -- a solver embedded in a host code that
// pre-reserves all device memory up front, code that runs while a CUDA graph
// is being captured elsewhere on the device, or real-time loops where an
// allocation could stall -- but still want the norm computed on the GPU.
//
// The scratch array is file-scope, so every GPU that loads this library holds
// it (kScratchBlocks * 4 doubles = 64 KiB) until the process exits, and every
// call on a device shares it: two calls whose kernels overlap on the GPU (for
// example on two streams) race on it and may return wrong norms.  Each call
// writes every partial it later reads, so nothing needs clearing between calls.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/tensum_gpu.h"

namespace {

constexpr int kThreads = 256;
constexpr int kScratchBlocks = 2048;       // partial-sum slots: 2048 blocks x 4 components
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_norm_scratch[kScratchBlocks * 4];

// Host-side record of the scratch array's device address, looked up once per device.
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {nullptr};

__global__ void k_norm_noalloc_part(const double* __restrict__ res, const double* __restrict__ area,
                                    const double* __restrict__ weight, int nv, double* __restrict__ part) {
  // grid-stride over vertices; the reference sums pow(residual/area, 2) * w per component
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
    const double a = area[i], w = weight[i];
    const double* r = res + 5 * (size_t)i;   // Flux layout: mass, mx, my, mz, energy
    double q0 = r[0] / a, q1 = r[1] / a, q2 = r[2] / a, q3 = r[4] / a;
    acc[0] += q0 * q0 * w;
    acc[1] += q1 * q1 * w;
    acc[2] += q2 * q2 * w;
    acc[3] += q3 * q3 * w;
  }
  __shared__ double red[4][kThreads];
#pragma unroll
  for (int c = 0; c < 4; ++c) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int o = kThreads / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
#pragma unroll
      for (int c = 0; c < 4; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int c = 0; c < 4; ++c) part[(size_t)blockIdx.x * 4 + c] = red[c][0];
}

__global__ void k_norm_noalloc_final(const double* __restrict__ part, int nblocks, int nv, double total0_in,
                                     double* __restrict__ out6) {
  __shared__ double red[4][kThreads];
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[c] += part[(size_t)b * 4 + c];
#pragma unroll
  for (int c = 0; c < 4; ++c) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int o = kThreads / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
#pragma unroll
      for (int c = 0; c < 4; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double n0 = sqrt(red[0][0]) / nv, n1 = sqrt(red[1][0]) / nv, n2 = sqrt(red[2][0]) / nv, n3 = sqrt(red[3][0]) / nv;
    double total = sqrt(n0 * n0 + (n1 * n1 + n2 * n2 + 0.0) + n3 * n3);
    // total0_in <= 0 marks the first iteration: the total becomes the normaliser (src/fv.cc:1860-1873)
    double total0 = total0_in > 0.0 ? total0_in : (total == 0.0 ? 1.0 : total);
    out6[0] = n0; out6[1] = n1; out6[2] = n2; out6[3] = n3;
    out6[4] = total / total0;
    out6[5] = total0;
  }
}

thread_local std::string g_err;

tg_status noalloc_fail(tg_status st, const char* msg, cudaError_t e = cudaSuccess) {
  g_err = msg;
  if (e != cudaSuccess) {
    g_err += ": ";
    g_err += cudaGetErrorString(e);
  }
  return st;
}

}  // namespace

extern "C" {

const char* tg_noalloc_last_error(void) { return g_err.c_str(); }

tg_status tg_residual_norm_noalloc(const double* res_dev, const double* dcarea_dev, const double* weight_dev,
                                   int n_vertex, double total0, double* out6_dev, void* stream) {
  if (!res_dev || !dcarea_dev || !weight_dev || !out6_dev)
    return noalloc_fail(TG_INVALID_ARG, "tg_residual_norm_noalloc: NULL buffer");
  if (n_vertex <= 0 || n_vertex > TG_NOALLOC_MAX_VERTICES)
    return noalloc_fail(TG_INVALID_ARG,
                        "tg_residual_norm_noalloc: n_vertex must be in 1..TG_NOALLOC_MAX_VERTICES (268435456)");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(TG_NO_DEVICE, "tg_residual_norm_noalloc: no current device", e);
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(TG_NOT_SUPPORTED, "tg_residual_norm_noalloc: device index too large");
  double* scratch = nullptr;
  {
    // first call on a device: look up the device address of the scratch array
    // (in host code its name is only a host-side stand-in)
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_norm_scratch);
      if (e != cudaSuccess) return noalloc_fail(TG_CUDA_ERROR, "tg_residual_norm_noalloc: cudaGetSymbolAddress", e);
      g_scratch_addr[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch_addr[dev];
  }
  int nblocks = (n_vertex + kThreads - 1) / kThreads;
  if (nblocks > kScratchBlocks) nblocks = kScratchBlocks;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_norm_noalloc_part<<<nblocks, kThreads, 0, s>>>(res_dev, dcarea_dev, weight_dev, n_vertex, scratch);
  k_norm_noalloc_final<<<1, kThreads, 0, s>>>(scratch, nblocks, n_vertex, total0, out6_dev);
  e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(TG_CUDA_ERROR, "tg_residual_norm_noalloc: launch", e);
  return TG_OK;
}

}  // extern "C"
