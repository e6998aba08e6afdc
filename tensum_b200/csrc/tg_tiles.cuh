// tg_tiles.cuh -- tiled stage kernels of the FP64 single-solve path.
//
// A tile is a contiguous range of owned vertices (Hilbert order) plus every
// vertex one edge away (periodic copies' neighbourhoods included).  One CTA
// per tile stages the tile's vertex data in shared memory once, so that
//   * each vertex's derived quantities (density, beta, entropy variables,
//     sound speed, logs) are evaluated once per staged copy instead of once
//     per incident edge, and
//   * each edge flux is computed once per tile into shared memory and summed
//     per owned vertex in a fixed order (deterministic, no flux buffer in HBM).
//
// k_tile_grad   compute_gradients (src/fv.cc:699-1059) for the owned vertices;
//               at the first stage of a step it also evaluates the local time
//               step (src/fv.cc:1499-1598) and U_old (src/fv.cc:1626-1630).
// k_tile_flux   compute_inviscid_residual + residual assembly
//               (src/fv.cc:1066-1192, 1467-1494) and, in MODE_UPDATE, the
//               SSP-RK3 update (src/fv.cc:1641-1652) with the residual norm
//               partial sums; writes the new state into the next buffer.
#pragma once

#include "tg_kernels.cuh"

namespace tg {

struct TileView {
  const int *vbeg, *loff, *eoff, *lv;
  const unsigned int* ab;
  const double *nx, *ny, *g0x, *g0y, *g1x, *g1y;
  const double *ux, *uy, *ar;   // unit normal and |n| per tile edge
  const int* cv_off;
  const unsigned short* cv_ent;
  const double *x, *y;    // vertex coordinates (device order)
};

constexpr int kTileThreads = 256;

__device__ __forceinline__ unsigned long long block_min_u64(unsigned long long bits) {
  bits = warp_min_u64(bits);
  __shared__ unsigned long long wmin[kTileThreads / 32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) wmin[w] = bits;
  __syncthreads();
  if (w == 0) {
    bits = lane < (int)(blockDim.x >> 5) ? wmin[lane] : 0x7ff0000000000000ull;
    bits = warp_min_u64(bits);
  }
  return bits;
}

// Gradients of the owned vertices; FIRST also computes dt and U_old.
template <bool FIRST>
__global__ void __launch_bounds__(kTileThreads) k_tile_grad(Params k, MeshView m, TileView t, StateView s,
                                                            Scalars* sc, const int* __restrict__ done) {
  if (*done) return;
  extern __shared__ double sm[];
  const int tile = blockIdx.x;
  const int l0 = t.loff[tile], L = t.loff[tile + 1] - l0;
  const int e0 = t.eoff[tile];
  const int nv = m.nv;
  double* sW = sm;              // 4 * L
  double* sU = sm + 4 * L;      // FIRST: u, v, c (3 * L)
  for (int i = threadIdx.x; i < L; i += blockDim.x) {
    int g = t.lv[l0 + i];
#pragma unroll
    for (int c = 0; c < 4; ++c) sW[c * L + i] = s.W[c * nv + g];
    if (FIRST) {
      Prim q = load_prim(s.P, nv, g);
      sU[i] = q.u;
      sU[L + i] = q.v;
      sU[2 * L + i] = sound_speed(k, q);
    }
  }
  __syncthreads();
  const int v = t.vbeg[tile] + threadIdx.x;
  const bool own = v < t.vbeg[tile + 1];
  unsigned long long bits = 0x7ff0000000000000ull;
  if (own) {
    double acc[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] = 0.0;
    double lam = 0.0;
    for (int j = t.cv_off[v]; j < t.cv_off[v + 1]; ++j) {
      int ent = t.cv_ent[j];
      int le = e0 + (ent >> 1), side = ent & 1;
      unsigned int ab = t.ab[le];
      int la = ab & 0xffff, lb = ab >> 16;
      int self = side ? lb : la, other = side ? la : lb;
      double gx = side ? t.g1x[le] : t.g0x[le];
      double gy = side ? t.g1y[le] : t.g0y[le];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        double dW = sW[c * L + other] - sW[c * L + self];
        acc[2 * c] += gx * dW;
        acc[2 * c + 1] += gy * dW;
      }
      if (FIRST) {
        double nx = t.nx[le], ny = t.ny[le];
        double area = sqrt(nx * nx + ny * ny);
        lam += (fabs(sU[self] * nx + sU[L + self] * ny) + sU[2 * L + self] * area) * 1.0;
      }
    }
    for (int j = m.cb_off[v]; j < m.cb_off[v + 1]; ++j) {
      int ent = m.cb_ent[j];
      int type = ent & 3, idx = ent >> 2;
      if (type == 1) {
        double dW[4];
        bface_grad_corr(k, m, s, idx, dW);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          acc[2 * c] += m.b_nx[idx] * dW[c];
          acc[2 * c + 1] += m.b_ny[idx] * dW[c];
        }
      } else if (FIRST && type == 0) {
        int d = idx >> 1;
        int selfg = (idx & 1) ? m.b_v1[d] : m.b_v0[d];
        Prim q = load_prim(s.P, nv, selfg);
        double nx = m.b_nx[d], ny = m.b_ny[d];
        double area = sqrt(nx * nx + ny * ny);
        lam += 0.5 * (fabs(q.u * nx + q.v * ny) + sound_speed(k, q) * area);
      }
    }
    double f = m.inv6mc[v];
#pragma unroll
    for (int c = 0; c < 8; ++c) s.G[c * nv + v] = acc[c] * f;
    if (FIRST) {
      if (k.model == 1) {
        for (int j = t.cv_off[v]; j < t.cv_off[v + 1]; ++j) {
          int ent = t.cv_ent[j];
          int le = e0 + (ent >> 1), side = ent & 1;
          unsigned int ab = t.ab[le];
          int la = ab & 0xffff, lb = ab >> 16;
          int selfg = t.lv[l0 + (side ? lb : la)];
          int ga = t.lv[l0 + la], gb = t.lv[l0 + lb];
          Prim q = load_prim(s.P, nv, selfg);
          double nx = t.nx[le], ny = t.ny[le];
          double area = sqrt(nx * nx + ny * ny);
          double dx = t.x[gb] - t.x[ga], dy = t.y[gb] - t.y[ga];
          double dl = sqrt(dx * dx + dy * dy);
          lam += (viscosity(k, q.T) * area / dl / density(k, q)) * 1.0;
        }
      }
      double dtv = k.cfl * m.dcarea[v] / lam;
      s.dt[v] = dtv;
      bits = (unsigned long long)__double_as_longlong(dtv);
      if (!(dtv > 0.0)) bits = 0x7ff0000000000000ull;
      Cons c = prim2con(k, load_prim(s.P, nv, v));
      s.Uold[v] = c.r; s.Uold[nv + v] = c.mx; s.Uold[2 * nv + v] = c.my; s.Uold[3 * nv + v] = c.E;
    }
  }
  if (FIRST) {
    bits = block_min_u64(bits);
    if (threadIdx.x == 0) atomicMin(&sc->dtmin_bits, bits);
  }
}

enum : int { MODE_RESIDUAL = 0, MODE_UPDATE = 1 };

// Shared-memory layout of one staged vertex (doubles, structure of arrays).
constexpr int kVRecFields = 8;   // rho u v p beta V1 a b
constexpr int kFluxSmemPerVertex = kVRecFields + 8 + 2;   // + gradient + coordinates

template <int FLUX, int RECON, int MODE>
__global__ void __launch_bounds__(kTileThreads) k_tile_flux(Params k, MeshView m, TileView t, StateView s,
                                                            Control ctl, Scalars* sc, int r, int do_norm,
                                                            double* __restrict__ Pout, double* __restrict__ Wout,
                                                            const int* __restrict__ done) {
  if (*done) return;
  extern __shared__ double sm[];
  const int tile = blockIdx.x;
  const int l0 = t.loff[tile], L = t.loff[tile + 1] - l0;
  const int e0 = t.eoff[tile], NE = t.eoff[tile + 1] - e0;
  const int nv = m.nv;
  constexpr bool kGrad = (FLUX == FLUX_TECNO_ROE || FLUX == FLUX_TECNO_RUSANOV) && RECON != RECON_FIRST;
  double* sV = sm;                          // kVRecFields * L
  double* sG = sm + kVRecFields * L;        // 8 * L
  double* sX = sG + 8 * L;                  // 2 * L
  double* sF = sX + 2 * L;                  // 4 * NE
  for (int i = threadIdx.x; i < L; i += blockDim.x) {
    int g = t.lv[l0 + i];
    VRec q = make_vrec<FLUX>(k, load_prim(s.P, nv, g));
    sV[0 * L + i] = q.rho; sV[1 * L + i] = q.u; sV[2 * L + i] = q.v; sV[3 * L + i] = q.p;
    sV[4 * L + i] = q.beta; sV[5 * L + i] = q.V1; sV[6 * L + i] = q.a; sV[7 * L + i] = q.b;
    if (kGrad) {
#pragma unroll
      for (int c = 0; c < 8; ++c) sG[c * L + i] = s.G[c * nv + g];
      sX[i] = t.x[g];
      sX[L + i] = t.y[g];
    }
  }
  __syncthreads();
  for (int le = threadIdx.x; le < NE; le += blockDim.x) {
    unsigned int ab = t.ab[e0 + le];
    int la = ab & 0xffff, lb = ab >> 16;
    VRec A, B;
    A.rho = sV[la]; A.u = sV[L + la]; A.v = sV[2 * L + la]; A.p = sV[3 * L + la];
    A.beta = sV[4 * L + la]; A.V1 = sV[5 * L + la]; A.a = sV[6 * L + la]; A.b = sV[7 * L + la];
    B.rho = sV[lb]; B.u = sV[L + lb]; B.v = sV[2 * L + lb]; B.p = sV[3 * L + lb];
    B.beta = sV[4 * L + lb]; B.V1 = sV[5 * L + lb]; B.a = sV[6 * L + lb]; B.b = sV[7 * L + lb];
    double gl[8], gr[8], dx = 0.0, dy = 0.0;
    if (kGrad) {
#pragma unroll
      for (int c = 0; c < 8; ++c) { gl[c] = sG[c * L + la]; gr[c] = sG[c * L + lb]; }
      dx = sX[lb] - sX[la];
      dy = sX[L + lb] - sX[L + la];
    }
    Flx F = num_flux_unit<FLUX, RECON>(k, A, B, t.ux[e0 + le], t.uy[e0 + le], t.ar[e0 + le], dx, dy, gl, gr);
    sF[le] = F.m; sF[NE + le] = F.x; sF[2 * NE + le] = F.y; sF[3 * NE + le] = F.e;
  }
  __syncthreads();
  const int v = t.vbeg[tile] + threadIdx.x;
  const bool own = v < t.vbeg[tile + 1];
  double nrm[4] = {0.0, 0.0, 0.0, 0.0};
  if (own) {
    double r0 = 0.0, r1 = 0.0, r2 = 0.0, r3 = 0.0;
    for (int j = t.cv_off[v]; j < t.cv_off[v + 1]; ++j) {
      int ent = t.cv_ent[j];
      int le = ent >> 1;
      double sg = (ent & 1) ? -1.0 : 1.0;
      r0 += sF[le] * sg; r1 += sF[NE + le] * sg; r2 += sF[2 * NE + le] * sg; r3 += sF[3 * NE + le] * sg;
    }
    const int n2 = 2 * m.nb, n3 = 3 * m.nvu;
    for (int j = m.cb_off[v]; j < m.cb_off[v + 1]; ++j) {
      int ent = m.cb_ent[j];
      int type = ent & 3, idx = ent >> 2;
      if (type == 0) {
        r0 += s.Fb[idx] * 0.5; r1 += s.Fb[n2 + idx] * 0.5; r2 += s.Fb[2 * n2 + idx] * 0.5; r3 += s.Fb[3 * n2 + idx] * 0.5;
      } else if (type == 2 && k.model == 1) {
        r1 += s.Fv[idx] * -(0.5 * 1.0); r2 += s.Fv[n3 + idx] * -(0.5 * 1.0); r3 += s.Fv[2 * n3 + idx] * -(0.5 * 1.0);
      } else if (type == 3 && k.model == 1) {
        r1 += s.Fvb[idx] * 0.5; r2 += s.Fvb[m.nb + idx] * 0.5; r3 += s.Fvb[2 * m.nb + idx] * 0.5;
      }
    }
    if (MODE == MODE_RESIDUAL) {
      s.R[v] = r0; s.R[nv + v] = r1; s.R[2 * nv + v] = r2; s.R[3 * nv + v] = r3;
    } else {
      const double a_rk[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0};
      const double b_rk[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
      double area = m.dcarea[v];
      if (do_norm) {
        double w = m.pweight[v];
        double q0 = r0 / area, q1 = r1 / area, q2 = r2 / area, q3 = r3 / area;
        nrm[0] = q0 * q0 * w; nrm[1] = q1 * q1 * w; nrm[2] = q2 * q2 * w; nrm[3] = q3 * q3 * w;
      }
      double dtv = (ctl.time_mode == 1 || ctl.time_step > 0.0) ? sc->dt_global : s.dt[v];
      double factor = dtv / (1.0 * area);
      Prim q0 = load_prim(s.P, nv, v);
      Cons c = prim2con(k, q0);
      double br = b_rk[r], ar = a_rk[r], c2 = -factor * br;
      c.r *= br; c.mx *= br; c.my *= br; c.E *= br;
      c.r += s.Uold[v] * ar + r0 * c2;
      c.mx += s.Uold[nv + v] * ar + r1 * c2;
      c.my += s.Uold[2 * nv + v] * ar + r2 * c2;
      c.E += s.Uold[3 * nv + v] * ar + r3 * c2;
      Prim q = con2prim(k, c);
      Ent e = prim2ent(k, q);
      Pout[v] = q.T; Pout[nv + v] = q.u; Pout[2 * nv + v] = q.v; Pout[3 * nv + v] = q.p;
      Wout[v] = e.f; Wout[nv + v] = e.vx; Wout[2 * nv + v] = e.vy; Wout[3 * nv + v] = e.l;
      bool ok = isfinite(q.T) && isfinite(q.u) && isfinite(q.v) && isfinite(q.p) && q.p > 0.0 && c.r > 0.0;
      if (!ok) atomicOr(&sc->bad, 1);
    }
  }
  if (MODE == MODE_UPDATE && do_norm) {
    // the smem tile buffers are no longer needed: reuse them for the block reduction
    __syncthreads();
    double* red = sm;
#pragma unroll
    for (int c = 0; c < 4; ++c) red[c * kTileThreads + threadIdx.x] = nrm[c];
    __syncthreads();
    for (int o = kTileThreads / 2; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o)
#pragma unroll
        for (int c = 0; c < 4; ++c) red[c * kTileThreads + threadIdx.x] += red[c * kTileThreads + threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0)
#pragma unroll
      for (int c = 0; c < 4; ++c) s.part[(size_t)blockIdx.x * 4 + c] = red[c * kTileThreads];
  }
}

inline size_t tile_grad_smem(int lmax, bool first) { return (size_t)lmax * (first ? 7 : 4) * sizeof(double); }
inline size_t tile_flux_smem(int lmax, int emax) {
  size_t a = ((size_t)lmax * kFluxSmemPerVertex + 4 * (size_t)emax) * sizeof(double);
  size_t b = 4 * kTileThreads * sizeof(double);
  return a > b ? a : b;
}

}  // namespace tg
