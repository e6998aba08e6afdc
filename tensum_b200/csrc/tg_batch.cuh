// tg_batch.cuh -- batched FP32 Monte Carlo ensembles: physics and kernels.
//
// An ensemble level is S samples of one periodic mesh, advanced together.
// Every per-sample array is [vertex or edge][component][sample] with the
// sample index innermost, so the 32 lanes of a warp hold 32 samples of one
// vertex: state loads are 128-byte coalesced, all components of a vertex are
// reached from one base address by immediate offsets, and the mesh data of the
// vertex and of its edges is read once per warp (a broadcast).  Members are FP32; geometry is
// formed in FP64 on the host and stored in FP32, the near-equal branch of the
// logarithmic mean is evaluated in FP64, and the per-sample clock (elapsed
// time, dt) is FP64 so output times are met exactly.
//
// Each stage is an edge pass (one flux per edge and sample, stored
// [component][edge][sample]) and a vertex pass that gathers the fluxes of the
// vertex's edges in a fixed order and applies the SSP-RK3 stage update: every
// flux is computed once, an edge's flux enters both endpoints bit for bit
// (exact conservation), and there are no atomics.
#pragma once

#include <cstdint>

#include "tg_physics.cuh"

namespace tg {
namespace batch {

constexpr int kMaxLevels = 4;
constexpr int kQ = 5;        // stored per vertex-sample: u, v, p, V1, V5
constexpr int kG = 8;        // dV1/dx, dV1/dy, dV2/dx, dV2/dy, dV3/dx, dV3/dy, dV5/dx, dV5/dy

// Mesh of one level (device order of the single-solve layout, tg_mesh.cc).
struct LevelMesh {
  int nv, ne;
  const int *e_a, *e_b;            // edge endpoints
  const float *ux, *uy, *ar;       // unit dual normal and |n| (formed in FP64)
  const float *nx, *ny;            // dual normal (for the time step)
  const float *dx, *dy;            // x_b - x_a
  const float *g0x, *g0y, *g1x, *g1y;   // P1 gradient weights of the a / b side
  const int *ce_off, *ce_ent;      // per-vertex gather: (edge << 1) | side
  const float *area, *inv6mc;      // dual area, 1 / (6 median area)
  const double* aw;                // dual area x periodic-copy weight (integrals)
  const double *x, *y;             // coordinates (initial conditions)
};

// Per-sample clock of one level.
struct LevelClock {
  double* elapsed;
  double* dt;
  unsigned int* dtmin_bits;        // FP32 bit pattern of the running min (positive floats order as uints)
  int* counter;
  int* reached;
  int* active;
  int* bad;
};

struct Level {
  LevelMesh m;
  LevelClock c;
  int S;                           // samples (a multiple of 32)
  int P;                           // row pitch in floats: S plus a pad that breaks power-of-two strides
  float* Q[3];                     // rotating states, nv x kQ x S
  float* Uold;                     // nv x 4 x S
  float* G;                        // nv x kG x S
  float* F;                        // ne x 4 x S: area-weighted edge fluxes of the current stage
  long long w_begin;               // first warp of this level in a fused launch (set per launch shape)
};

struct Batch {
  int nlev;
  Level lev[kMaxLevels];
  long long work;                  // warps of a fused launch over all levels
};

struct BParams {
  float gamma, R, inv_gm1, inv_gamma, sqrt_gm1, cfl, ev_alpha, ev_beta;
  double final_time;
  const double* tinst;
  int ntinst;
  int stop_counter;                // unused on the device: the live value is *stop
  const int* stop;                 // samples hold once their output counter exceeds it
  int flux, recon;
};

// -------------------------------------------------------------- FP32 physics
struct FRec { float rho, u, v, p, beta, V1, a; };
struct FFlx { float m, x, y, e; };

// Ismail-Roe logarithmic mean F (logmean = (a+b)/2 / F) with the near-equal
// series branch in FP64 (src/material.h:24-42).
// 1 / d from the FP32 reciprocal refined by one Newton-Raphson step,
// y1 = y0 (2 - d y0): relative error 2^-24 -> about 2^-46, ample for FP32
// inputs, in three FP64 operations instead of a full FP64 division.
__device__ __forceinline__ double recip_nr(double d) {
  const double y = (double)__frcp_rn((float)d);
  return y * (2.0 - d * y);
}

__device__ __forceinline__ float logavg_F_mixed(float a, float b) {
  const double da = a, db = b;
  const double f = (db - da) * recip_nr(db + da);   // b - a and b + a are exact in FP64
  const double u = f * f;
  if (u < 1.0e-2) {
    const double u2 = u * u;
    return (float)(1.0 + u * (1.0 / 3.0) + u2 * (1.0 / 5.0) + u2 * u * (1.0 / 7.0));
  }
  return logf(b / a) / (2.0f * (float)f);
}

__device__ __forceinline__ FRec frec(const BParams& k, float u, float v, float p, float V1, float V5, bool need_a) {
  FRec r;
  r.rho = -V5 * p;          // V5 = -2 beta, beta = rho / (2 p)
  r.u = u; r.v = v; r.p = p;
  r.beta = -0.5f * V5;
  r.V1 = V1;
  r.a = need_a ? sqrtf(k.gamma * p / r.rho) : 0.0f;
  return r;
}

__device__ __forceinline__ float fminmod(float a, float b) {      // src/limiter.h:14-27
  if (a < 0.0f && b < 0.0f) return -fminf(-a, -b);
  if (a > 0.0f && b > 0.0f) return fminf(a, b);
  return 0.0f;
}

// Z_ji - Z_ij for first order / minmod reconstruction (src/reconstruct.cc:139-188)
template <int RECON>
__device__ __forceinline__ float fjump(float d, float gl, float gr) {
  if (RECON == RECON_FIRST) return d;
  return d - 0.5f * fminmod(2.0f * gr - d, d) - 0.5f * fminmod(2.0f * gl - d, d);
}

// KEPEC central flux (src/kepec.cc:10-38) on a unit normal.
__device__ __forceinline__ FFlx fkepec(const BParams& k, const FRec& L, const FRec& R, float unx, float uny,
                                       float& rho_ln, float& ibeta) {
  // __fdividef: at most 2 ulp for the magnitudes of densities and beta
  rho_ln = __fdividef(0.5f * (L.rho + R.rho), logavg_F_mixed(L.rho, R.rho));
  ibeta = __fdividef(logavg_F_mixed(L.beta, R.beta), 0.5f * (L.beta + R.beta));
  const float p = __fdividef(0.5f * (L.rho + R.rho), L.beta + R.beta);
  const float vx = 0.5f * (L.u + R.u), vy = 0.5f * (L.v + R.v);
  const float vn = vx * unx + vy * uny;
  const float vel2 = 0.5f * ((L.u * L.u + L.v * L.v) + (R.u * R.u + R.v * R.v));
  FFlx F;
  F.m = rho_ln * vn;
  F.x = unx * p + vx * F.m;
  F.y = uny * p + vy * F.m;
  F.e = 0.5f * (ibeta * k.inv_gm1 - vel2) * F.m + (F.x * vx + F.y * vy);
  return F;
}

// KEPES-TeCNO (src/kepes_tecno_roe.cc:11-173, src/kepes_tecno_rusanov.cc:11-164):
// KEPEC minus 0.5 R Lambda (Z_ji - Z_ij), R applied through its column structure.
template <int ROE, int RECON>
__device__ __forceinline__ FFlx ftecno(const BParams& k, const FRec& L, const FRec& R, float unx, float uny, float dx,
                                       float dy, const float* gL, const float* gR) {
  float rho, ibeta;
  FFlx F = fkepec(k, L, R, unx, uny, rho, ibeta);
  const float a = sqrtf(0.5f * k.gamma * ibeta);
  const float p = __fdividef(0.5f * (L.rho + R.rho), L.beta + R.beta);
  const float vx = 0.5f * (L.u + R.u), vy = 0.5f * (L.v + R.v);
  const float vn = vx * unx + vy * uny;
  const float vsq = vx * vx + vy * vy;
  const float H = a * a * k.inv_gm1 + 0.5f * vsq;
  const float v1 = vx * uny - vy * unx;
  const float c1 = sqrtf(rho * k.inv_gamma);
  const float S0 = 0.70710678118654752f * c1, S1 = k.sqrt_gm1 * c1, S2 = sqrtf(p);
  auto RT = [&](const float* x, float* z) {
    const float A = x[0] + vx * x[1] + vy * x[2];
    const float B = unx * x[1] + uny * x[2] + vn * x[3];
    const float C = A + H * x[3];
    z[0] = S0 * (C - a * B);
    z[1] = S1 * (A + (0.5f * vsq) * x[3]);
    z[2] = S2 * (uny * x[1] - unx * x[2] + v1 * x[3]);
    z[3] = S0 * (C + a * B);
  };
  float Lam[4];
  if (ROE) {
    const float vnl = L.u * unx + L.v * uny, vnr = R.u * unx + R.v * uny;
    Lam[0] = (1.0f + k.ev_beta) * fabsf(vn - a) + k.ev_alpha * fabsf((vnl - L.a) - (vnr - R.a));
    Lam[1] = Lam[2] = fabsf(vn);
    Lam[3] = (1.0f + k.ev_beta) * fabsf(vn + a) + k.ev_alpha * fabsf((vnl + L.a) - (vnr + R.a));
  } else {
    Lam[0] = Lam[1] = Lam[2] = Lam[3] = fabsf(vn) + fabsf(a);
  }
  // V = (V1, 2 beta u, 2 beta v, -2 beta)
  const float dV[4] = {R.V1 - L.V1, 2.0f * (R.u * R.beta - L.u * L.beta), 2.0f * (R.v * R.beta - L.v * L.beta),
                       -2.0f * (R.beta - L.beta)};
  float d[4], sl[4], sr[4];
  RT(dV, d);
  if (RECON != RECON_FIRST) {
    float gl[4], gr[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      gl[i] = gL[2 * i] * dx + gL[2 * i + 1] * dy;
      gr[i] = gR[2 * i] * dx + gR[2 * i + 1] * dy;
    }
    RT(gl, sl);
    RT(gr, sr);
  }
  float q[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) q[i] = Lam[i] * fjump<RECON>(d[i], RECON != RECON_FIRST ? sl[i] : 0.0f,
                                                             RECON != RECON_FIRST ? sr[i] : 0.0f);
  q[0] *= S0; q[1] *= S1; q[2] *= S2; q[3] *= S0;
  const float sum = q[0] + q[1] + q[3], dif = q[3] - q[0];
  F.m -= 0.5f * sum;
  F.x -= 0.5f * (vx * sum + a * unx * dif + uny * q[2]);
  F.y -= 0.5f * (vy * sum + a * uny * dif - unx * q[2]);
  F.e -= 0.5f * (H * (q[0] + q[3]) + a * vn * dif + (0.5f * vsq) * q[1] + v1 * q[2]);
  return F;
}

template <int FLUX, int RECON>
__device__ __forceinline__ FFlx fflux(const BParams& k, const FRec& L, const FRec& R, float unx, float uny, float dx,
                                      float dy, const float* gL, const float* gR) {
  if (FLUX == FLUX_TECNO_ROE) return ftecno<1, RECON>(k, L, R, unx, uny, dx, dy, gL, gR);
  if (FLUX == FLUX_TECNO_RUSANOV) return ftecno<0, RECON>(k, L, R, unx, uny, dx, dy, gL, gR);
  float r, b;
  return fkepec(k, L, R, unx, uny, r, b);
}

// ------------------------------------------------------------------ indexing
// A warp covers 32/ST vertices x ST samples (the sample tile ST is 32 or 16);
// warps are ordered sample-group-major, so consecutive warps walk neighbouring
// vertices of one sample group and the group's states stay in L2 while its
// neighbours are read.
struct Item { int l, v, s; bool ok; };

template <int ST>
__host__ __device__ __forceinline__ long long level_warps(int nv, int S) {
  constexpr int VPW = 32 / ST;
  return (long long)((nv + VPW - 1) / VPW) * (S / ST);
}

// EDGE: items are (edge, sample) instead of (vertex, sample).
template <int ST, bool EDGE = false>
__device__ __forceinline__ Item item_of(const Batch& B, long long w, int lane) {
  constexpr int VPW = 32 / ST;
  Item it{0, 0, 0, false};
  if (w >= B.work) return it;
  int l = 0;
#pragma unroll
  for (int i = 1; i < kMaxLevels; ++i)
    if (i < B.nlev && w >= B.lev[i].w_begin) l = i;
  const long long r = w - B.lev[l].w_begin;
  const int n = EDGE ? B.lev[l].m.ne : B.lev[l].m.nv;
  const int nvw = (n + VPW - 1) / VPW;
  it.l = l;
  it.s = (int)(r / nvw) * ST + (lane % ST);
  it.v = (int)(r % nvw) * VPW + lane / ST;
  it.ok = it.v < n;
  return it;
}

// Row block of item i in a [item][C][sample] array (add the sample, then c * S).
__device__ __forceinline__ size_t rows(int i, int C, int S) { return (size_t)i * C * S; }

// -------------------------------------------------------------------- kernels
// Per-sample step start: which samples advance, reset of the running dt min.
__global__ void kb_step_begin(Batch B, BParams k) {
  const int l = blockIdx.y;
  if (l >= B.nlev) return;
  const Level& L = B.lev[l];
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= L.S) return;
  const bool go = !L.c.bad[s] && L.c.elapsed[s] < k.final_time && L.c.counter[s] <= *k.stop;
  L.c.active[s] = go ? 1 : 0;
  L.c.dtmin_bits[s] = 0x7f800000u;
}

// Local time step (src/fv.cc:1499-1580, inviscid) of every vertex and the
// running per-sample minimum; U_old (src/fv.cc:1626-1630).  Each thread keeps
// one sample and walks a strided set of vertices, so one atomic per block and
// sample remains.
template <int VT>
__global__ void __launch_bounds__(32 * VT) kb_dt(Batch B, BParams k, int chunks) {
  const int lane = threadIdx.x & 31, vg = threadIdx.x >> 5;
  // blockIdx.x: (level, sample group, chunk)
  long long bid = blockIdx.x;
  int l = 0;
  long long base = 0;
  for (int i = 0; i < B.nlev; ++i) {
    const long long nb = (long long)(B.lev[i].S >> 5) * chunks;
    if (bid < base + nb) { l = i; break; }
    base += nb;
  }
  const Level& L = B.lev[l];
  const long long r = bid - base;
  const int sg = (int)(r / chunks), ch = (int)(r % chunks);
  const int s = sg * 32 + lane;
  const bool act = L.c.active[s];
  float m = __int_as_float(0x7f800000);
  if (act) {
    const int per = (L.m.nv + chunks - 1) / chunks;
    const int v0 = ch * per, v1 = min(L.m.nv, v0 + per);
    for (int v = v0 + vg; v < v1; v += VT) {
      const float* q = L.Q[0] + rows(v, kQ, L.P) + s;
      const float u = q[0], w = q[L.P], p = q[2 * L.P], V5 = q[4 * L.P];
      const float rho = -V5 * p;
      const float c = sqrtf(k.gamma * p / rho);
      float lam = 0.0f;
      for (int j = L.m.ce_off[v]; j < L.m.ce_off[v + 1]; ++j) {
        const int e = L.m.ce_ent[j] >> 1;
        const float nx = L.m.nx[e], ny = L.m.ny[e];
        lam += fabsf(u * nx + w * ny) + c * L.m.ar[e];
      }
      const float dtv = k.cfl * L.m.area[v] / lam;
      m = fminf(m, dtv > 0.0f ? dtv : __int_as_float(0x7f800000));
      // U_old
      float* uo = L.Uold + rows(v, 4, L.P) + s;
      uo[0] = rho;
      uo[L.P] = rho * u;
      uo[2 * L.P] = rho * w;
      uo[3 * L.P] = p * k.inv_gm1 + 0.5f * (u * u + w * w) * rho;
    }
  }
  __shared__ float red[VT][32];
  red[vg][lane] = m;
  __syncthreads();
  if (vg == 0) {
    for (int i = 1; i < VT; ++i) m = fminf(m, red[i][lane]);
    if (act) atomicMin(&L.c.dtmin_bits[s], __float_as_uint(m));
  }
}

// Global dt per sample and the clamp to its next output time (src/fv.cc:1584-1618).
__global__ void kb_dt_final(Batch B, BParams k) {
  const int l = blockIdx.y;
  if (l >= B.nlev) return;
  const Level& L = B.lev[l];
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= L.S || !L.c.active[s]) return;
  double dtg = (double)__uint_as_float(L.c.dtmin_bits[s]);
  const int c = L.c.counter[s] < k.ntinst ? L.c.counter[s] : k.ntinst - 1;
  if (L.c.elapsed[s] + dtg > k.tinst[c]) {
    dtg = k.tinst[c] - L.c.elapsed[s];
    L.c.reached[s] = 1;
  }
  L.c.dt[s] = dtg;
}

// Gradients of the entropy variables (src/fv.cc:699-1059 in the edge form
// grad_v = sum_e g_{v,e} (W_o - W_v) / (6 mcarea)), one (vertex, sample) per thread.
template <int ST>
__global__ void kb_grad(Batch B, BParams k, int r) {
  const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const Item it = item_of<ST>(B, w, threadIdx.x & 31);
  if (!it.ok) return;
  const Level& L = B.lev[it.l];
  if (!L.c.active[it.s]) return;
  const int v = it.v, s = it.s;
  const int S = L.P;   // row pitch
  const float* Q = L.Q[r] + s;
  auto W = [&](int x, float* o) {
    const float* q = Q + rows(x, kQ, S);
    const float u = q[0], vv = q[S], V5 = q[4 * S];
    o[0] = q[3 * S]; o[1] = -V5 * u; o[2] = -V5 * vv; o[3] = V5;   // V2 = 2 beta u = -V5 u
  };
  float ws[4];
  W(v, ws);
  float acc[kG];
#pragma unroll
  for (int c = 0; c < kG; ++c) acc[c] = 0.0f;
  for (int j = L.m.ce_off[v]; j < L.m.ce_off[v + 1]; ++j) {
    const int ent = L.m.ce_ent[j], e = ent >> 1, side = ent & 1;
    const int o = side ? L.m.e_a[e] : L.m.e_b[e];
    const float gx = side ? L.m.g1x[e] : L.m.g0x[e], gy = side ? L.m.g1y[e] : L.m.g0y[e];
    float wo[4];
    W(o, wo);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const float d = wo[c] - ws[c];
      acc[2 * c] += gx * d;
      acc[2 * c + 1] += gy * d;
    }
  }
  const float f = L.m.inv6mc[v];
  float* G = L.G + rows(v, kG, S) + s;
#pragma unroll
  for (int c = 0; c < kG; ++c) G[c * S] = acc[c] * f;
}

// Edge fluxes of one stage (src/fv.cc:1066-1192, src/material.cc:27-74): one
// (edge, sample) per thread, the flux of the edge's own orientation (a left,
// b right) times |n|, stored for the gather.  Held samples skip.
template <int FLUX, int RECON, int ST, int BS>
__global__ void __launch_bounds__(BS) kb_edge_flux(Batch B, BParams k, int r) {
  const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const Item it = item_of<ST, true>(B, w, threadIdx.x & 31);
  if (!it.ok) return;
  const Level& L = B.lev[it.l];
  const int e = it.v, s = it.s;
  if (!L.c.active[s]) return;
  constexpr bool kA = (FLUX == FLUX_TECNO_ROE);
  constexpr bool kGr = (RECON != RECON_FIRST) && (FLUX == FLUX_TECNO_ROE || FLUX == FLUX_TECNO_RUSANOV);
  const int S = L.P;   // row pitch
  const int ia = L.m.e_a[e], ib = L.m.e_b[e];
  const float* qa = L.Q[r] + rows(ia, kQ, S) + s;
  const float* qb = L.Q[r] + rows(ib, kQ, S) + s;
  const FRec A = frec(k, qa[0], qa[S], qa[2 * S], qa[3 * S], qa[4 * S], kA);
  const FRec Bv = frec(k, qb[0], qb[S], qb[2 * S], qb[3 * S], qb[4 * S], kA);
  float ga[kG], gb[kG];
  if (kGr) {
    const float* Ga = L.G + rows(ia, kG, S) + s;
    const float* Gb = L.G + rows(ib, kG, S) + s;
#pragma unroll
    for (int c = 0; c < kG; ++c) { ga[c] = Ga[c * S]; gb[c] = Gb[c * S]; }
  }
  const FFlx F = fflux<FLUX, RECON>(k, A, Bv, L.m.ux[e], L.m.uy[e], L.m.dx[e], L.m.dy[e], ga, gb);
  const float ar = L.m.ar[e];
  float* Fo = L.F + rows(e, 4, S) + s;
  Fo[0] = F.m * ar; Fo[S] = F.x * ar; Fo[2 * S] = F.y * ar; Fo[3 * S] = F.e * ar;
}

// Residual gather in the fixed per-vertex edge order and the SSP-RK3 stage
// update (src/fv.cc:1635-1658), state r -> state (r+1) % 3.  Held or finished
// samples copy their state through.
template <int ST, int BS>
__global__ void __launch_bounds__(BS) kb_gather_update(Batch B, BParams k, int r) {
  const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const Item it = item_of<ST>(B, w, threadIdx.x & 31);
  if (!it.ok) return;
  const Level& L = B.lev[it.l];
  const int v = it.v, s = it.s;
  const int S = L.P;   // row pitch
  const size_t ov = rows(v, kQ, S) + s;
  const float* Q = L.Q[r] + ov;
  float* Qn = L.Q[(r + 1) % 3] + ov;
  if (!L.c.active[s]) {
#pragma unroll
    for (int c = 0; c < kQ; ++c) Qn[c * S] = Q[c * S];
    return;
  }
  float r0 = 0.0f, r1 = 0.0f, r2 = 0.0f, r3 = 0.0f;
  const int j0 = L.m.ce_off[v], j1 = L.m.ce_off[v + 1];
#pragma unroll 4
  for (int j = j0; j < j1; ++j) {
    const int ent = L.m.ce_ent[j];
    const float* Fe = L.F + rows(ent >> 1, 4, S) + s;
    const float sg = (ent & 1) ? -1.0f : 1.0f;
    r0 += Fe[0] * sg; r1 += Fe[S] * sg; r2 += Fe[2 * S] * sg; r3 += Fe[3 * S] * sg;
  }
  const float u0 = Q[0], v0 = Q[S], p0 = Q[2 * S], V50 = Q[4 * S];
  const float rho0 = -V50 * p0;
  // Shu-Osher SSP-RK3 stage (src/constants.h:4-6)
  const float a_rk = r == 0 ? 0.0f : (r == 1 ? 0.75f : 1.0f / 3.0f);
  const float b_rk = r == 0 ? 1.0f : (r == 1 ? 0.25f : 2.0f / 3.0f);
  const float factor = (float)L.c.dt[s] / L.m.area[v];
  const float c2 = -factor * b_rk;
  const float* Uo = L.Uold + rows(v, 4, S) + s;
  const float cr = rho0 * b_rk + Uo[0] * a_rk + r0 * c2;
  const float cx = rho0 * u0 * b_rk + Uo[S] * a_rk + r1 * c2;
  const float cy = rho0 * v0 * b_rk + Uo[2 * S] * a_rk + r2 * c2;
  const float cE = (p0 * k.inv_gm1 + 0.5f * (u0 * u0 + v0 * v0) * rho0) * b_rk + Uo[3 * S] * a_rk + r3 * c2;
  const float ir = 1.0f / cr;
  const float u = cx * ir, vv = cy * ir;
  const float p = (k.gamma - 1.0f) * (cE - 0.5f * (cx * u + cy * vv));
  const float beta = 0.5f * cr / p;
  const float sent = logf(p) - k.gamma * logf(cr);
  const float V1 = (k.gamma - sent) * k.inv_gm1 - (u * u + vv * vv) * beta;
  Qn[0] = u;
  Qn[S] = vv;
  Qn[2 * S] = p;
  Qn[3 * S] = V1;
  Qn[4 * S] = -2.0f * beta;
  if (!(p > 0.0f) || !(cr > 0.0f) || !isfinite(u) || !isfinite(vv) || !isfinite(p)) L.c.bad[s] = 1;
}

// Per-sample step end (src/fv.cc:2307-2336).
__global__ void kb_step_end(Batch B, BParams k) {
  const int l = blockIdx.y;
  if (l >= B.nlev) return;
  const Level& L = B.lev[l];
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= L.S || !L.c.active[s]) return;
  L.c.elapsed[s] += L.c.dt[s];
  if (L.c.reached[s]) {
    L.c.counter[s] += 1;
    L.c.reached[s] = 0;
  }
}

// Initial states of Kelvin-Helmholtz samples from their random-number rows
// (the parameter-file condition with pert(4, ...), src/perturb.cc:196-208):
// v' = 0.01 sum_k r_k sin(2 pi k x + 2 pi r_{M+k}), evaluated in FP64.
__global__ void kb_ic_kh(Level L, BParams k, const double* __restrict__ rnd, int nrnd) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)L.m.nv * L.S) return;
  const int v = (int)(t / L.S), s = (int)(t % L.S);
  const double x = L.m.x[v], y = L.m.y[v];
  const double* row = rnd + (size_t)s * nrnd;
  const int M = nrnd / 2;
  const double two_pi = 6.283185307179586;
  double acc = 0.0;
  for (int i = 1; i <= M; ++i) acc = acc + row[i - 1] * sin(two_pi * i * x + two_pi * row[M + i - 1]);
  const bool inside = fabs(y - 0.5) < 0.25;
  const double rho = inside ? 2.0 : 1.0, p = 2.5, u = inside ? 0.5 : -0.5, vv = 0.01 * acc;
  const double beta = rho / (2.0 * p);
  const double sent = log(p) - (double)k.gamma * log(rho);
  const double V1 = ((double)k.gamma - sent) / ((double)k.gamma - 1.0) - (u * u + vv * vv) * beta;
  float* q = L.Q[0] + rows(v, kQ, L.P) + s;
  q[0] = (float)u;
  q[L.P] = (float)vv;
  q[2 * L.P] = (float)p;
  q[3 * L.P] = (float)V1;
  q[4 * L.P] = (float)(-2.0 * beta);
}

// Ensemble moments of one level at its current state, FP64: Welford mean and
// sum of squared deviations in sample order (the per-group recurrence of
// increment_moments, src/fv.cc:595-694) and a Kahan-compensated sum of
// squares.  One thread per (component, vertex); record layout as
// tg_moments_*: PrimVar (T, p, u, v, w), then density, mach, entropy.
__global__ void kb_moments(Level L, BParams k, int extras, int nvar, double* __restrict__ fm, double* __restrict__ sm,
                           double* __restrict__ m2) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nvar * L.m.nv) return;
  const int c = (int)(t / L.m.nv), v = (int)(t % L.m.nv);
  // which derived quantity component c is
  int kind = c;   // 0 T, 1 p, 2 u, 3 v, 4 w, 5+ extras in bit order
  if (c >= 5) {
    int want = c - 5, b = 0;
    for (; b < 4; ++b)
      if ((extras >> b) & 1) { if (want == 0) break; --want; }
    kind = 5 + b;
  }
  double mean = 0.0, ssd = 0.0, sq = 0.0, comp = 0.0;
  for (int s = 0; s < L.S; ++s) {
    const float* q = L.Q[0] + rows(v, kQ, L.P) + s;
    const double u = q[0], w = q[L.P], p = q[2 * L.P];
    const double V5 = q[4 * L.P];
    const double rho = -V5 * p;
    double x;
    switch (kind) {
      case 0: x = p / ((double)k.R * rho); break;
      case 1: x = p; break;
      case 2: x = u; break;
      case 3: x = w; break;
      case 4: x = 0.0; break;
      case 5: x = rho; break;
      case 6: x = sqrt(u * u + w * w) / sqrt((double)k.gamma * p / rho); break;
      default: x = log(p) - (double)k.gamma * log(rho); break;
    }
    const double kk = (double)(s + 1);
    const double prev = mean;
    mean = s == 0 ? x : (c < 5 ? x * (1.0 / kk) + prev * ((kk - 1.0) / kk) : prev + (x - prev) / kk);
    if (s > 0) ssd += (x - prev) * (x - mean);
    const double y = x * x - comp;       // Kahan
    const double tsum = sq + y;
    comp = (tsum - sq) - y;
    sq = tsum;
  }
  const size_t o = (size_t)c * L.m.nv + v;
  fm[o] = mean;
  sm[o] = sq;
  m2[o] = ssd;
}

// Per-sample integrals (FP64) of one level's current states, the
// compute_global quantities (src/fv.cc:2186-2203) plus the vertical kinetic
// energy: q0 = sum 0.5 rho v^2 A w, q1 = sum 0.5 rho u^2 A w,
// q2 = sum -rho s / (gamma - 1) A w.  Block (sample group, vertex chunk);
// partial[chunk][sample][3], summed over chunks in order by the host.
template <int VT>
__global__ void __launch_bounds__(32 * VT) kb_integrals(Level L, BParams k, int chunks, double* __restrict__ partial) {
  const int lane = threadIdx.x & 31, vg = threadIdx.x >> 5;
  const int sg = blockIdx.x / chunks, ch = blockIdx.x % chunks;
  const int s = sg * 32 + lane;
  const int per = (L.m.nv + chunks - 1) / chunks;
  const int v0 = ch * per, v1 = min(L.m.nv, v0 + per);
  double q[3] = {0.0, 0.0, 0.0};
  for (int v = v0 + vg; v < v1; v += VT) {
    const float* r = L.Q[0] + rows(v, kQ, L.P) + s;
    const double u = r[0], w = r[L.P], p = r[2 * L.P], V5 = r[4 * L.P];
    const double rho = -V5 * p;
    const double aw = L.m.aw[v];
    q[0] += 0.5 * rho * w * w * aw;
    q[1] += 0.5 * rho * u * u * aw;
    q[2] += -rho * (log(p) - (double)k.gamma * log(rho)) / ((double)k.gamma - 1.0) * aw;
  }
  __shared__ double red[3][VT][32];
#pragma unroll
  for (int c = 0; c < 3; ++c) red[c][vg][lane] = q[c];
  __syncthreads();
  if (vg == 0) {
    for (int i = 1; i < VT; ++i)
#pragma unroll
      for (int c = 0; c < 3; ++c) q[c] += red[c][i][lane];
#pragma unroll
    for (int c = 0; c < 3; ++c) partial[((size_t)ch * L.S + s) * 3 + c] = q[c];
  }
}

}  // namespace batch
}  // namespace tg
