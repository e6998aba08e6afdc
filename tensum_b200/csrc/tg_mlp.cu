// tg_mlp.cu -- the surrogate network of the multi-fidelity Monte Carlo estimator.
//
// A fixed-shape multilayer perceptron din -> 64 -> 64 -> 64 -> dout with GELU
// (0.5 x (1 + erf(x / sqrt 2))) after each hidden layer, trained in FP32 by
// full forward / backward passes written here (mean squared error, Adam), and
// evaluated in BF16 on the tensor cores for the large surrogate sample sets.
// The network only ever serves as a control variate; it has no counterpart in
// the reference.
//
// Parameters are one FP32 vector: W1[64][din] b1[64] W2[64][64] b2[64]
// W3[64][64] b3[64] W4[dout][64] b4[dout] (W[out][in], row major).
// Every reduction over the batch runs in a fixed order (one thread per weight
// sums its samples in sequence), so training is bitwise reproducible.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/tensum_gpu.h"

namespace {

constexpr int H = 64;
constexpr int kMaxIn = 32;
constexpr int kMaxOut = 8;
thread_local std::string g_mlp_error;

struct Offs {
  int w1, b1, w2, b2, w3, b3, w4, b4, n;
};

__host__ __device__ inline Offs offsets(int din, int dout) {
  Offs o;
  o.w1 = 0; o.b1 = o.w1 + H * din;
  o.w2 = o.b1 + H; o.b2 = o.w2 + H * H;
  o.w3 = o.b2 + H; o.b3 = o.w3 + H * H;
  o.w4 = o.b3 + H; o.b4 = o.w4 + dout * H;
  o.n = o.b4 + dout;
  return o;
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float x) {
  // d/dx [x Phi(x)] = Phi(x) + x phi(x)
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.3989422804014327f * expf(-0.5f * x * x);
}

// Forward pass of one sample per thread; keeps the pre-activations z1..z3 and
// the outputs for the backward pass.  Parameters are staged in shared memory.
__global__ void k_forward(const float* __restrict__ theta, int din, int dout, const float* __restrict__ X, int n,
                          float* __restrict__ Z, float* __restrict__ Y) {
  extern __shared__ float sp[];
  const Offs o = offsets(din, dout);
  for (int i = threadIdx.x; i < o.n; i += blockDim.x) sp[i] = theta[i];
  __syncthreads();
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  float a[H], z[H];
  float x[kMaxIn];
  for (int i = 0; i < din; ++i) x[i] = X[(size_t)b * din + i];
  for (int j = 0; j < H; ++j) {
    float s = sp[o.b1 + j];
    for (int i = 0; i < din; ++i) s = fmaf(sp[o.w1 + j * din + i], x[i], s);
    z[j] = s;
  }
  for (int j = 0; j < H; ++j) { Z[((size_t)b * 3 + 0) * H + j] = z[j]; a[j] = gelu(z[j]); }
  const int wl[2] = {o.w2, o.w3}, bl[2] = {o.b2, o.b3};
  for (int l = 0; l < 2; ++l) {
    for (int j = 0; j < H; ++j) {
      float s = sp[bl[l] + j];
#pragma unroll 16
      for (int i = 0; i < H; ++i) s = fmaf(sp[wl[l] + j * H + i], a[i], s);
      z[j] = s;
    }
    for (int j = 0; j < H; ++j) { Z[((size_t)b * 3 + 1 + l) * H + j] = z[j]; a[j] = gelu(z[j]); }
  }
  for (int j = 0; j < dout; ++j) {
    float s = sp[o.b4 + j];
#pragma unroll 16
    for (int i = 0; i < H; ++i) s = fmaf(sp[o.w4 + j * H + i], a[i], s);
    Y[(size_t)b * dout + j] = s;
  }
}

// Per-sample deltas of the mean squared error L = sum (y - t)^2 / (n dout):
// D[b][0..2] are dL/dz of the three hidden layers, D4 dL/dy.
__global__ void k_deltas(const float* __restrict__ theta, int din, int dout, const float* __restrict__ Z,
                         const float* __restrict__ Y, const float* __restrict__ T, int n, float* __restrict__ D,
                         float* __restrict__ D4) {
  extern __shared__ float sp[];
  const Offs o = offsets(din, dout);
  for (int i = threadIdx.x; i < o.n; i += blockDim.x) sp[i] = theta[i];
  __syncthreads();
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  float d4[kMaxOut];
  const float scale = 2.0f / ((float)n * (float)dout);
  for (int j = 0; j < dout; ++j) {
    d4[j] = (Y[(size_t)b * dout + j] - T[(size_t)b * dout + j]) * scale;
    D4[(size_t)b * dout + j] = d4[j];
  }
  float d[H], dn[H];
  for (int i = 0; i < H; ++i) {
    float s = 0.0f;
    for (int j = 0; j < dout; ++j) s = fmaf(sp[o.w4 + j * H + i], d4[j], s);
    d[i] = s * gelu_d(Z[((size_t)b * 3 + 2) * H + i]);
  }
  for (int i = 0; i < H; ++i) D[((size_t)b * 3 + 2) * H + i] = d[i];
  const int wl[2] = {o.w3, o.w2};
  for (int l = 0; l < 2; ++l) {
    const int zl = 1 - l;
    for (int i = 0; i < H; ++i) {
      float s = 0.0f;
#pragma unroll 16
      for (int j = 0; j < H; ++j) s = fmaf(sp[wl[l] + j * H + i], d[j], s);
      dn[i] = s * gelu_d(Z[((size_t)b * 3 + zl) * H + i]);
    }
    for (int i = 0; i < H; ++i) { d[i] = dn[i]; D[((size_t)b * 3 + zl) * H + i] = d[i]; }
  }
}

// One thread per parameter: its gradient summed over the batch in sample order.
__global__ void k_grads(int din, int dout, const float* __restrict__ X, const float* __restrict__ Z,
                        const float* __restrict__ D, const float* __restrict__ D4, int n, float* __restrict__ g) {
  const Offs o = offsets(din, dout);
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= o.n) return;
  float s = 0.0f;
  if (p < o.b1) {                                  // W1[j][i]: sum d1[j] x[i]
    const int j = p / din, i = p % din;
    for (int b = 0; b < n; ++b) s = fmaf(D[((size_t)b * 3 + 0) * H + j], X[(size_t)b * din + i], s);
  } else if (p < o.w2) {                           // b1[j]
    const int j = p - o.b1;
    for (int b = 0; b < n; ++b) s += D[((size_t)b * 3 + 0) * H + j];
  } else if (p < o.b2 || (p >= o.w3 && p < o.b3)) {  // W2 / W3: sum d[j] gelu(z_prev[i])
    const bool l3 = p >= o.w3;
    const int q = p - (l3 ? o.w3 : o.w2), j = q / H, i = q % H;
    const int dl = l3 ? 2 : 1, zl = l3 ? 1 : 0;
    for (int b = 0; b < n; ++b)
      s = fmaf(D[((size_t)b * 3 + dl) * H + j], gelu(Z[((size_t)b * 3 + zl) * H + i]), s);
  } else if (p < o.w3 || (p >= o.b3 && p < o.w4)) {  // b2 / b3
    const bool l3 = p >= o.b3;
    const int j = p - (l3 ? o.b3 : o.b2), dl = l3 ? 2 : 1;
    for (int b = 0; b < n; ++b) s += D[((size_t)b * 3 + dl) * H + j];
  } else if (p < o.b4) {                           // W4[j][i]: sum d4[j] gelu(z3[i])
    const int q = p - o.w4, j = q / H, i = q % H;
    for (int b = 0; b < n; ++b) s = fmaf(D4[(size_t)b * dout + j], gelu(Z[((size_t)b * 3 + 2) * H + i]), s);
  } else {                                         // b4[j]
    const int j = p - o.b4;
    for (int b = 0; b < n; ++b) s += D4[(size_t)b * dout + j];
  }
  g[p] = s;
}

// Adam (Kingma & Ba, 2015) with bias correction.
__global__ void k_adam(int np, float* __restrict__ theta, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const float gp = g[p];
  const float mp = b1 * m[p] + (1.0f - b1) * gp;
  const float vp = b2 * v[p] + (1.0f - b2) * gp * gp;
  m[p] = mp;
  v[p] = vp;
  theta[p] -= lr * (mp / c1) / (sqrtf(vp / c2) + eps);
}

__global__ void k_loss(const float* __restrict__ Y, const float* __restrict__ T, int n, int dout, float* out) {
  __shared__ float red[256];
  float s = 0.0f;
  for (int i = threadIdx.x; i < n * dout; i += blockDim.x) {
    const float d = Y[i] - T[i];
    s = fmaf(d, d, s);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0] / ((float)n * (float)dout);
}

// ---------------------------------------------------------------- BF16 inference
// Each warp takes 16 samples; a hidden layer is the 16 x 64 activation tile
// times W^T (64 x 64) on the tensor cores: 8 column tiles of 8 x 4 k-steps of
// mma.sync.m16n8k16 (BF16 in, FP32 accumulate).  Fragment ownership follows the
// PTX ISA layout of m16n8k16: with g = lane / 4 and t = lane % 4, A rows g and
// g + 8, columns 2t, 2t+1 (+8); B (k x n) rows 2t, 2t+1 (+8), column g; C rows
// g, g + 8, columns 2t, 2t + 1.
__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<unsigned*>(&v);
}

__device__ __forceinline__ void mma_bf16(float* c, const unsigned* a, const unsigned* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

constexpr int kInferWarps = 4;

__global__ void __launch_bounds__(32 * kInferWarps)
    k_infer_bf16(const float* __restrict__ theta, int din, int dout, const float* __restrict__ X, int n,
                 float* __restrict__ Y) {
  __shared__ __nv_bfloat16 sw[2][H * H];           // W2, W3 in BF16, [out][in]
  __shared__ float sf[H * kMaxIn + H * kMaxOut + 4 * H + kMaxOut];
  __shared__ float act[kInferWarps][16][H + 4];      // per-warp activation tile (FP32, padded)
  const Offs o = offsets(din, dout);
  for (int i = threadIdx.x; i < H * H; i += blockDim.x) {
    sw[0][i] = __float2bfloat16_rn(theta[o.w2 + i]);
    sw[1][i] = __float2bfloat16_rn(theta[o.w3 + i]);
  }
  float* w1 = sf;
  float* w4 = w1 + H * kMaxIn;
  float* bias = w4 + H * kMaxOut;                    // b1, b2, b3, b4
  for (int i = threadIdx.x; i < H * din; i += blockDim.x) w1[i] = theta[o.w1 + i];
  for (int i = threadIdx.x; i < dout * H; i += blockDim.x) w4[i] = theta[o.w4 + i];
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    bias[i] = theta[o.b1 + i]; bias[H + i] = theta[o.b2 + i]; bias[2 * H + i] = theta[o.b3 + i];
  }
  for (int i = threadIdx.x; i < dout; i += blockDim.x) bias[3 * H + i] = theta[o.b4 + i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  float(*A)[H + 4] = act[warp];
  const long long tiles = ((long long)n + 15) / 16;
  for (long long tile = (long long)blockIdx.x * kInferWarps + warp; tile < tiles;
       tile += (long long)gridDim.x * kInferWarps) {
    const long long base = tile * 16;
    // layer 1 in FP32 (din is small): lane handles rows r = lane / 2 ... two lanes per row
    for (int e = lane; e < 16 * H; e += 32) {
      const int r = e / H, j = e % H;
      const long long b = base + r;
      float s = bias[j];
      if (b < n)
        for (int i = 0; i < din; ++i) s = fmaf(w1[j * din + i], X[b * din + i], s);
      A[r][j] = gelu(s);
    }
    __syncwarp();
    for (int l = 0; l < 2; ++l) {
      const __nv_bfloat16* W = sw[l];
      float c[8][4];
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) c[nt][0] = c[nt][1] = c[nt][2] = c[nt][3] = 0.0f;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        const int k0 = ks * 16;
        unsigned a[4];
        a[0] = pack_bf16(A[g][k0 + 2 * t], A[g][k0 + 2 * t + 1]);
        a[1] = pack_bf16(A[g + 8][k0 + 2 * t], A[g + 8][k0 + 2 * t + 1]);
        a[2] = pack_bf16(A[g][k0 + 2 * t + 8], A[g][k0 + 2 * t + 9]);
        a[3] = pack_bf16(A[g + 8][k0 + 2 * t + 8], A[g + 8][k0 + 2 * t + 9]);
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
          // B[k][n] = W[n][k]: column n = nt * 8 + g, rows k0 + 2t, +1 and +8, +9
          const __nv_bfloat16* wr = W + (nt * 8 + g) * H + k0 + 2 * t;
          unsigned b[2];
          b[0] = *reinterpret_cast<const unsigned*>(wr);
          b[1] = *reinterpret_cast<const unsigned*>(wr + 8);
          mma_bf16(c[nt], a, b);
        }
      }
      __syncwarp();
      const float* bl = bias + (l + 1) * H;
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const int col = nt * 8 + 2 * t;
        A[g][col] = gelu(c[nt][0] + bl[col]);
        A[g][col + 1] = gelu(c[nt][1] + bl[col + 1]);
        A[g + 8][col] = gelu(c[nt][2] + bl[col]);
        A[g + 8][col + 1] = gelu(c[nt][3] + bl[col + 1]);
      }
      __syncwarp();
    }
    // output layer in FP32
    for (int e = lane; e < 16 * dout; e += 32) {
      const int r = e / dout, j = e % dout;
      const long long b = base + r;
      if (b >= n) continue;
      float s = bias[3 * H + j];
      for (int i = 0; i < H; ++i) s = fmaf(w4[j * H + i], A[r][i], s);
      Y[b * dout + j] = s;
    }
    __syncwarp();
  }
}

}  // namespace

struct tg_mlp {
  int din = 0, dout = 0, np = 0;
  long long step = 0;
  cudaStream_t stream = nullptr;
  float *theta = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;
  // training scratch, grown on demand
  int cap = 0;
  float *X = nullptr, *T = nullptr, *Z = nullptr, *Y = nullptr, *D = nullptr, *D4 = nullptr, *loss = nullptr;
  std::string err;
};

namespace {

tg_status mfail(tg_mlp* h, tg_status st, const std::string& msg) {
  if (h) h->err = msg;
  g_mlp_error = msg;
  return st;
}

#define TM_CUDA(h, call)                                                                          \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      return mfail((h), TG_CUDA_ERROR, std::string(#call " failed: ") + cudaGetErrorString(e_)); \
  } while (0)

tg_status reserve(tg_mlp* h, int n) {
  if (n <= h->cap) return TG_OK;
  cudaFree(h->X); cudaFree(h->T); cudaFree(h->Z); cudaFree(h->Y); cudaFree(h->D); cudaFree(h->D4);
  h->X = h->T = h->Z = h->Y = h->D = h->D4 = nullptr;
  h->cap = 0;
  TM_CUDA(h, cudaMalloc((void**)&h->X, (size_t)n * h->din * sizeof(float)));
  TM_CUDA(h, cudaMalloc((void**)&h->T, (size_t)n * h->dout * sizeof(float)));
  TM_CUDA(h, cudaMalloc((void**)&h->Y, (size_t)n * h->dout * sizeof(float)));
  TM_CUDA(h, cudaMalloc((void**)&h->D4, (size_t)n * h->dout * sizeof(float)));
  TM_CUDA(h, cudaMalloc((void**)&h->Z, (size_t)n * 3 * H * sizeof(float)));
  TM_CUDA(h, cudaMalloc((void**)&h->D, (size_t)n * 3 * H * sizeof(float)));
  h->cap = n;
  return TG_OK;
}

size_t param_smem(const tg_mlp* h) { return (size_t)h->np * sizeof(float); }

// forward + deltas + parameter gradients of one batch already in h->X, h->T
void enqueue_grad(tg_mlp* h, int n) {
  const int blk = 128, nb = (n + blk - 1) / blk;
  k_forward<<<nb, blk, param_smem(h), h->stream>>>(h->theta, h->din, h->dout, h->X, n, h->Z, h->Y);
  k_deltas<<<nb, blk, param_smem(h), h->stream>>>(h->theta, h->din, h->dout, h->Z, h->Y, h->T, n, h->D, h->D4);
  k_grads<<<(h->np + 127) / 128, 128, 0, h->stream>>>(h->din, h->dout, h->X, h->Z, h->D, h->D4, n, h->g);
  k_loss<<<1, 256, 0, h->stream>>>(h->Y, h->T, n, h->dout, h->loss);
}

}  // namespace

extern "C" {

tg_status tg_mlp_create(int din, int dout, unsigned long long seed, tg_mlp** out) {
  if (!out) return mfail(nullptr, TG_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (din < 1 || din > kMaxIn || dout < 1 || dout > kMaxOut)
    return mfail(nullptr, TG_INVALID_ARG, "din must be 1..32 and dout 1..8");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return mfail(nullptr, TG_NO_DEVICE, "no CUDA device visible; the GPU path has no CPU fallback");
  tg_mlp* h = new (std::nothrow) tg_mlp();
  if (!h) return mfail(nullptr, TG_INVALID_ARG, "out of host memory");
  h->din = din; h->dout = dout;
  h->np = offsets(din, dout).n;
  // He-style uniform initialisation from a 64-bit linear congruential stream (Knuth's MMIX constants)
  std::vector<float> th(h->np, 0.0f);
  const Offs o = offsets(din, dout);
  unsigned long long st = seed * 6364136223846793005ULL + 1442695040888963407ULL;
  auto uni = [&]() {
    st = st * 6364136223846793005ULL + 1442695040888963407ULL;
    return (double)(st >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](int off, int rows, int cols) {
    const double a = std::sqrt(6.0 / cols);
    for (int i = 0; i < rows * cols; ++i) th[off + i] = (float)((2.0 * uni() - 1.0) * a);
  };
  fill(o.w1, H, din); fill(o.w2, H, H); fill(o.w3, H, H); fill(o.w4, dout, H);
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->theta, h->np * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->m, h->np * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->v, h->np * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->g, h->np * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->loss, sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(h->theta, th.data(), h->np * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(h->m, 0, h->np * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(h->v, 0, h->np * sizeof(float));
  if (e != cudaSuccess) {
    tg_mlp_destroy(h);
    return mfail(nullptr, TG_CUDA_ERROR, cudaGetErrorString(e));
  }
  *out = h;
  return TG_OK;
}

tg_status tg_mlp_destroy(tg_mlp* h) {
  if (!h) return TG_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  cudaFree(h->theta); cudaFree(h->m); cudaFree(h->v); cudaFree(h->g); cudaFree(h->loss);
  cudaFree(h->X); cudaFree(h->T); cudaFree(h->Z); cudaFree(h->Y); cudaFree(h->D); cudaFree(h->D4);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return TG_OK;
}

const char* tg_mlp_last_error(const tg_mlp* h) { return h ? h->err.c_str() : g_mlp_error.c_str(); }

int tg_mlp_n_params(const tg_mlp* h) { return h ? h->np : 0; }

tg_status tg_mlp_get_params(tg_mlp* h, float* theta) {
  if (!h || !theta) return mfail(h, TG_INVALID_ARG, "NULL argument");
  TM_CUDA(h, cudaMemcpyAsync(theta, h->theta, h->np * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  TM_CUDA(h, cudaStreamSynchronize(h->stream));
  return TG_OK;
}

tg_status tg_mlp_set_params(tg_mlp* h, const float* theta) {
  if (!h || !theta) return mfail(h, TG_INVALID_ARG, "NULL argument");
  TM_CUDA(h, cudaMemcpyAsync(h->theta, theta, h->np * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  TM_CUDA(h, cudaMemsetAsync(h->m, 0, h->np * sizeof(float), h->stream));
  TM_CUDA(h, cudaMemsetAsync(h->v, 0, h->np * sizeof(float), h->stream));
  TM_CUDA(h, cudaStreamSynchronize(h->stream));
  h->step = 0;
  return TG_OK;
}

// Loss and parameter gradient of one batch (host arrays), for gradient checks.
tg_status tg_mlp_loss_grad(tg_mlp* h, const float* X, const float* T, int n, float* loss, float* grad) {
  if (!h || !X || !T || n < 1) return mfail(h, TG_INVALID_ARG, "bad batch");
  tg_status st = reserve(h, n);
  if (st != TG_OK) return st;
  TM_CUDA(h, cudaMemcpyAsync(h->X, X, (size_t)n * h->din * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  TM_CUDA(h, cudaMemcpyAsync(h->T, T, (size_t)n * h->dout * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  enqueue_grad(h, n);
  TM_CUDA(h, cudaGetLastError());
  if (loss) TM_CUDA(h, cudaMemcpyAsync(loss, h->loss, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  if (grad) TM_CUDA(h, cudaMemcpyAsync(grad, h->g, h->np * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  TM_CUDA(h, cudaStreamSynchronize(h->stream));
  return TG_OK;
}

// Adam training on (X, T) (host arrays, n samples) in mini-batches taken in
// order, `epochs` passes.  losses (may be NULL) receives the last batch loss of
// every epoch.
tg_status tg_mlp_train(tg_mlp* h, const float* X, const float* T, int n, int epochs, int batch, float lr,
                       float* losses) {
  if (!h || !X || !T || n < 1 || epochs < 1 || batch < 1) return mfail(h, TG_INVALID_ARG, "bad training set");
  if (batch > n) batch = n;
  tg_status st = reserve(h, n);
  if (st != TG_OK) return st;
  float *dX = nullptr, *dT = nullptr;
  TM_CUDA(h, cudaMalloc((void**)&dX, (size_t)n * h->din * sizeof(float)));
  TM_CUDA(h, cudaMalloc((void**)&dT, (size_t)n * h->dout * sizeof(float)));
  TM_CUDA(h, cudaMemcpyAsync(dX, X, (size_t)n * h->din * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  TM_CUDA(h, cudaMemcpyAsync(dT, T, (size_t)n * h->dout * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  cudaError_t e = cudaSuccess;
  for (int ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
    for (int s0 = 0; s0 < n && e == cudaSuccess; s0 += batch) {
      const int nb = std::min(batch, n - s0);
      e = cudaMemcpyAsync(h->X, dX + (size_t)s0 * h->din, (size_t)nb * h->din * sizeof(float),
                          cudaMemcpyDeviceToDevice, h->stream);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(h->T, dT + (size_t)s0 * h->dout, (size_t)nb * h->dout * sizeof(float),
                            cudaMemcpyDeviceToDevice, h->stream);
      enqueue_grad(h, nb);
      ++h->step;
      const float c1 = 1.0f - std::pow(b1, (float)h->step), c2 = 1.0f - std::pow(b2, (float)h->step);
      k_adam<<<(h->np + 255) / 256, 256, 0, h->stream>>>(h->np, h->theta, h->g, h->m, h->v, lr, b1, b2, eps, c1, c2);
    }
    if (losses && e == cudaSuccess) e = cudaMemcpyAsync(losses + ep, h->loss, sizeof(float), cudaMemcpyDeviceToHost, h->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaFree(dX);
  cudaFree(dT);
  if (e != cudaSuccess) return mfail(h, TG_CUDA_ERROR, cudaGetErrorString(e));
  return TG_OK;
}

// Evaluation of n inputs (host or device arrays; device when on_device != 0):
// precision 0 = FP32 SIMT (the training path), 1 = BF16 tensor cores.
tg_status tg_mlp_predict(tg_mlp* h, const float* X, int n, float* Y, int precision, int on_device) {
  if (!h || !X || !Y || n < 1) return mfail(h, TG_INVALID_ARG, "bad prediction set");
  const float* dX = X;
  float* dY = Y;
  float* own = nullptr;
  if (!on_device) {
    TM_CUDA(h, cudaMalloc((void**)&own, (size_t)n * (h->din + h->dout) * sizeof(float)));
    TM_CUDA(h, cudaMemcpyAsync(own, X, (size_t)n * h->din * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    dX = own;
    dY = own + (size_t)n * h->din;
  }
  if (precision == 1) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    const long long tiles = ((long long)n + 15) / 16;
    const int grid = (int)std::min<long long>((tiles + kInferWarps - 1) / kInferWarps, 8LL * sms);
    k_infer_bf16<<<grid, 32 * kInferWarps, 0, h->stream>>>(h->theta, h->din, h->dout, dX, n, dY);
  } else {
    float* Z = nullptr;
    cudaError_t e = cudaMalloc((void**)&Z, (size_t)n * 3 * H * sizeof(float));
    if (e != cudaSuccess) { cudaFree(own); return mfail(h, TG_CUDA_ERROR, cudaGetErrorString(e)); }
    k_forward<<<(n + 127) / 128, 128, param_smem(h), h->stream>>>(h->theta, h->din, h->dout, dX, n, Z, dY);
    cudaStreamSynchronize(h->stream);
    cudaFree(Z);
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && !on_device)
    e = cudaMemcpyAsync(Y, dY, (size_t)n * h->dout * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(own);
  if (e != cudaSuccess) return mfail(h, TG_CUDA_ERROR, cudaGetErrorString(e));
  return TG_OK;
}

}  // extern "C"
