// tg_tiles.cuh -- tiled stage kernels of the FP64 single-solve path.
//
// A tile is a contiguous range of owned vertices (Hilbert order) plus every
// vertex one edge away (periodic copies' neighbourhoods included).  One CTA
// per tile stages everything the tile needs -- the gathered vertex data, the
// tile's edge arrays and the owned vertices' gather lists -- into shared
// memory with asynchronous copies issued all at once (cp.async), so a CTA has
// its whole working set in flight before it waits.  Then:
//   * each vertex's derived quantities (density, beta, entropy variables,
//     sound speed, logs) are evaluated once per staged copy instead of once
//     per incident edge,
//   * each edge flux is computed once per tile and written over the edge's own
//     (already consumed) geometry slots, and
//   * every owned vertex sums its edge fluxes in a fixed order
//     (deterministic; no flux buffer in HBM).
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

#ifndef TG_TILE_OWNED
#define TG_TILE_OWNED 128      // owned vertices per tile (<= kTileThreads)
#endif
#ifndef TG_TILE_LCAP
#define TG_TILE_LCAP 256       // local (owned + halo) vertices per tile
#endif
#ifndef TG_TILE_ECAP
#define TG_TILE_ECAP 512       // edges per tile
#endif
// resident flux CTAs per SM the register budget is sized for: TeCNO fluxes / central fluxes.
// Measured at KH 1025^2: 7 central / gradient CTAs (72 / 70 registers, a 48-byte spill in
// the update-mode central kernels) beat 6 (80 / 74 registers) by 5% a step, 8 (64
// registers, 100+ bytes of spills) lose; 5 TeCNO CTAs spill and lose.
#ifndef TG_FLUX_MINB
#define TG_FLUX_MINB 4
#endif
#ifndef TG_FLUX_MINB_CENTRAL
#define TG_FLUX_MINB_CENTRAL 7
#endif
#ifndef TG_GRAD_MINB
#define TG_GRAD_MINB 7         // resident gradient / dt CTAs per SM the register budget is sized for
#endif

namespace tg {

struct TileView {
  const int *vbeg, *loff, *eoff, *lv;
  const unsigned int* ab;
  const double *nx, *ny, *g0x, *g0y, *g1x, *g1y;
  const double *ux, *uy, *ar;   // unit normal and |n| per tile edge
  const double* r;              // radius per tile edge (axisymmetric runs)
  const int* cv_off;            // per vertex (nv + 1); cv_ent has an even length
  const unsigned short* cv_ent;
  const double *x, *y;          // vertex coordinates (device order)
  // ordered launches (ORD kernels: a partition's frontier or interior tiles): block b
  // works on tile order[base + b], and total counts the tiles of every launch of the
  // pass; the other kernels work on tile blockIdx.x over one launch of all tiles
  const int* order;
  int base, total;
};

template <bool ORD>
__device__ __forceinline__ int tile_of_block(const TileView& t) {
  return ORD ? t.order[t.base + blockIdx.x] : (int)blockIdx.x;
}

#ifndef TG_TILE_THREADS
#define TG_TILE_THREADS 128    // threads per tile CTA (>= TG_TILE_OWNED)
#endif
constexpr int kTileThreads = TG_TILE_THREADS;

// ---- asynchronous global -> shared copies (sm_80+ cp.async)
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

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

// Stage the owned vertices' gather lists: the entries, in whole 4-byte words
// from the even entry at or below the tile's first one (returned as the base
// the offsets are taken relative to), and the offsets.
__device__ __forceinline__ int stage_lists(const TileView& t, int vb, int nown, unsigned int* sC, int* sO) {
  const int base = t.cv_off[vb] & ~1;
  const int nwords = (t.cv_off[vb + nown] - base + 1) >> 1;
  const unsigned int* src = reinterpret_cast<const unsigned int*>(t.cv_ent + base);
  for (int i = threadIdx.x; i < nwords; i += blockDim.x) cp_async4(sC + i, src + i);
  for (int i = threadIdx.x; i <= nown; i += blockDim.x) cp_async4(sO + i, t.cv_off + vb + i);
  return base;
}

__device__ __forceinline__ int list_entry(const unsigned int* sC, int j) {
  return (int)((sC[j >> 1] >> ((j & 1) * 16)) & 0xffffu);
}

// ---------------------------------------------------------------- gradients
// Shared memory: W (4 per local vertex) [+ T, u, v at FIRST];
// per edge: gradient weights (4) [+ normal (2) at FIRST] + endpoints (4 bytes);
// gather lists.
__host__ __device__ constexpr int grad_vertex_doubles(bool first) { return first ? 7 : 4; }
__host__ __device__ constexpr int grad_edge_doubles(bool first) { return first ? 6 : 4; }

// warm_only (gradient kernels at a step's first stage): runs only when the
// previous step's last stage has already formed dt and U_old for this state,
// the first-stage kernel (FIRST) only when it has not.
template <bool FIRST, bool GRAD, bool ORD = false>
__global__ void __launch_bounds__(kTileThreads, TG_GRAD_MINB) k_tile_grad(Params k, MeshView m, TileView t, StateView s,
                                                            Scalars* sc, int lmax, int emax,
                                                            const int* __restrict__ done, int warm_only) {
  if (*done) return;
  const bool warm = k.fuse_dt && sc->dt_next;
  if ((FIRST && warm) || (warm_only && !warm)) return;
  const bool dt_here = FIRST;
  extern __shared__ double sm[];
  const int tile = tile_of_block<ORD>(t);
  const int l0 = t.loff[tile], L = t.loff[tile + 1] - l0;
  const int e0 = t.eoff[tile], NE = t.eoff[tile + 1] - e0;
  const int vb = t.vbeg[tile], nown = t.vbeg[tile + 1] - vb;
  const int nv = m.nv;
  double* sW = sm;                                   // 4 * L
  double* sU = sm + 4 * lmax;                        // FIRST: T, u, v -> c, u, v (3 * L)
  double* sE = sm + grad_vertex_doubles(FIRST) * lmax;   // g0x g0y g1x g1y [nx ny]
  unsigned int* sAB = reinterpret_cast<unsigned int*>(sE + grad_edge_doubles(FIRST) * emax);
  int* sO = reinterpret_cast<int*>(sAB + emax);      // nown + 1
  unsigned int* sC = reinterpret_cast<unsigned int*>(sO + kTileThreads + 2);

  for (int i = threadIdx.x; i < L; i += blockDim.x) {
    int g = t.lv[l0 + i];
    if (GRAD)
#pragma unroll
      for (int c = 0; c < 4; ++c) cp_async8(sW + c * L + i, s.W + (size_t)c * nv + g);
    if (dt_here) {
      cp_async8(sU + i, s.P + g);                              // T
      cp_async8(sU + L + i, s.P + (size_t)nv + g);             // u
      cp_async8(sU + 2 * L + i, s.P + (size_t)2 * nv + g);     // v
    }
  }
  for (int le = threadIdx.x; le < NE; le += blockDim.x) {
    if (GRAD) {
      cp_async8(sE + le, t.g0x + e0 + le);
      cp_async8(sE + NE + le, t.g0y + e0 + le);
      cp_async8(sE + 2 * NE + le, t.g1x + e0 + le);
      cp_async8(sE + 3 * NE + le, t.g1y + e0 + le);
    }
    if (dt_here) {
      cp_async8(sE + 4 * NE + le, t.nx + e0 + le);
      cp_async8(sE + 5 * NE + le, t.ny + e0 + le);
    }
    cp_async4(sAB + le, t.ab + e0 + le);
  }
  const int cbase = stage_lists(t, vb, nown, sC, sO);
  cp_async_wait_all();
  __syncthreads();
  if (dt_here) {
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
      Prim q;
      q.T = sU[i];
      sU[i] = sound_speed(k, q);
    }
    __syncthreads();
  }
  const int tid = threadIdx.x;
  const int v = vb + tid;
  unsigned long long bits = 0x7ff0000000000000ull;
  if (tid < nown) {
    double acc[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] = 0.0;
    double lam = 0.0;
    const int j0 = sO[tid] - cbase, j1 = sO[tid + 1] - cbase;
    for (int j = j0; j < j1; ++j) {
      int ent = list_entry(sC, j);
      int le = ent >> 1, side = ent & 1;
      unsigned int ab = sAB[le];
      int la = ab & 0xffff, lb = ab >> 16;
      int self = side ? lb : la, other = side ? la : lb;
      if (GRAD) {
        double gx = sE[(side ? 2 : 0) * NE + le];
        double gy = sE[(side ? 3 : 1) * NE + le];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          double dW = sW[c * L + other] - sW[c * L + self];
          acc[2 * c] += gx * dW;
          acc[2 * c + 1] += gy * dW;
        }
      }
      if (dt_here) {
        double nx = sE[4 * NE + le], ny = sE[5 * NE + le];
        double area = face_area(nx, ny);
        lam += face_radius(sU[L + self], sU[2 * L + self], nx, ny, sU[self], area) * 1.0;
      }
    }
    for (int j = m.cb_off[v]; j < m.cb_off[v + 1]; ++j) {
      int ent = m.cb_ent[j];
      int type = ent & 3, idx = ent >> 2;
      if (GRAD && type == 1) {
        double dW[4];
        bface_grad_corr(k, m, s, idx, dW);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          acc[2 * c] += m.b_nx[idx] * dW[c];
          acc[2 * c + 1] += m.b_ny[idx] * dW[c];
        }
      } else if (dt_here && type == 0) {
        int d = idx >> 1;
        int selfg = (idx & 1) ? m.b_v1[d] : m.b_v0[d];
        Prim q = load_prim(s.P, nv, selfg);
        double nx = m.b_nx[d], ny = m.b_ny[d];
        double area = face_area(nx, ny);
        lam += 0.5 * face_radius(q.u, q.v, nx, ny, sound_speed(k, q), area);
      }
    }
    if (GRAD) {
      double f = m.inv6mc[v];
#pragma unroll
      for (int c = 0; c < 8; ++c) s.G[(size_t)c * nv + v] = acc[c] * f;
    }
    if (dt_here) {
      if (k.model == 1) {
        for (int j = j0; j < j1; ++j) {
          int ent = list_entry(sC, j);
          int le = ent >> 1, side = ent & 1;
          unsigned int ab = sAB[le];
          int la = ab & 0xffff, lb = ab >> 16;
          int selfg = t.lv[l0 + (side ? lb : la)];
          int ga = t.lv[l0 + la], gb = t.lv[l0 + lb];
          Prim q = load_prim(s.P, nv, selfg);
          double nx = sE[4 * NE + le], ny = sE[5 * NE + le];
          double area = face_area(nx, ny);
          double dx = t.x[gb] - t.x[ga], dy = t.y[gb] - t.y[ga];
          double dl = face_area(dx, dy);
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
  if (dt_here) {
    bits = block_min_u64(bits);
    if (threadIdx.x == 0) atomicMin(&sc->dtmin_bits, bits);
  }
}

// --------------------------------------------------------------------- fluxes
enum : int { MODE_RESIDUAL = 0, MODE_UPDATE = 1 };

// Shared-memory slots of the per-vertex record fields each flux reads (-1:
// unused), and where the raw inputs are staged before the record is formed in
// place: p, u, v from P, the entropy variables V1 (W0) and V5 = -2 beta (W3)
// from W, and T where a sound speed is needed.
template <int FLUX> struct VLayout;
template <> struct VLayout<FLUX_TECNO_ROE> { enum { rho = 0, u = 1, v = 2, p = -1, beta = 3, V1 = 4, a = 5, b = -1, n = 6,
                                                    Rp = 0, Ru = 1, Rv = 2, RW3 = 3, RW0 = 4, RT = 5 }; };
template <> struct VLayout<FLUX_TECNO_RUSANOV> { enum { rho = 0, u = 1, v = 2, p = -1, beta = 3, V1 = 4, a = -1, b = -1, n = 5,
                                                        Rp = 0, Ru = 1, Rv = 2, RW3 = 3, RW0 = 4, RT = -1 }; };
template <> struct VLayout<FLUX_KEPEC> { enum { rho = 0, u = 1, v = 2, p = -1, beta = 3, V1 = -1, a = -1, b = -1, n = 4,
                                                Rp = 0, Ru = 1, Rv = 2, RW3 = 3, RW0 = -1, RT = -1 }; };
template <> struct VLayout<FLUX_KEP> { enum { rho = 0, u = 1, v = 2, p = 3, beta = -1, V1 = -1, a = 4, b = -1, n = 5,
                                              Rp = 3, Ru = 1, Rv = 2, RW3 = 0, RW0 = -1, RT = 4 }; };
template <> struct VLayout<FLUX_ROE_EC> { enum { rho = -1, u = 0, v = 1, p = 2, beta = -1, V1 = -1, a = -1, b = 3, n = 4,
                                                 Rp = 2, Ru = 0, Rv = 1, RW3 = 3, RW0 = -1, RT = -1 }; };
template <> struct VLayout<FLUX_AVG> { enum { rho = 0, u = 1, v = 2, p = 3, beta = -1, V1 = -1, a = -1, b = -1, n = 4,
                                              Rp = 3, Ru = 1, Rv = 2, RW3 = 0, RW0 = -1, RT = -1 }; };

template <int FLUX, int RECON>
__host__ __device__ constexpr bool flux_needs_grad() {
  return (FLUX == FLUX_TECNO_ROE || FLUX == FLUX_TECNO_RUSANOV) && RECON != RECON_FIRST;
}
// doubles per staged vertex: record fields [+ gradient (8) + coordinates (2)]
template <int FLUX, int RECON>
__host__ __device__ constexpr int flux_vertex_doubles() {
  return VLayout<FLUX>::n + (flux_needs_grad<FLUX, RECON>() ? 10 : 0);
}

template <int FLUX>
__device__ __forceinline__ void store_vrec(double* sV, int L, int i, const VRec& q) {
  typedef VLayout<FLUX> Y;
  if (Y::rho >= 0) sV[Y::rho * L + i] = q.rho;
  if (Y::u >= 0) sV[Y::u * L + i] = q.u;
  if (Y::v >= 0) sV[Y::v * L + i] = q.v;
  if (Y::p >= 0) sV[Y::p * L + i] = q.p;
  if (Y::beta >= 0) sV[Y::beta * L + i] = q.beta;
  if (Y::V1 >= 0) sV[Y::V1 * L + i] = q.V1;
  if (Y::a >= 0) sV[Y::a * L + i] = q.a;
  if (Y::b >= 0) sV[Y::b * L + i] = q.b;
}

template <int FLUX>
__device__ __forceinline__ VRec load_vrec(const double* sV, int L, int i) {
  typedef VLayout<FLUX> Y;
  VRec q;
  q.rho = Y::rho >= 0 ? sV[(Y::rho >= 0 ? Y::rho : 0) * L + i] : 0.0;
  q.u = Y::u >= 0 ? sV[(Y::u >= 0 ? Y::u : 0) * L + i] : 0.0;
  q.v = Y::v >= 0 ? sV[(Y::v >= 0 ? Y::v : 0) * L + i] : 0.0;
  q.p = Y::p >= 0 ? sV[(Y::p >= 0 ? Y::p : 0) * L + i] : 0.0;
  q.beta = Y::beta >= 0 ? sV[(Y::beta >= 0 ? Y::beta : 0) * L + i] : 0.0;
  q.V1 = Y::V1 >= 0 ? sV[(Y::V1 >= 0 ? Y::V1 : 0) * L + i] : 0.0;
  q.a = Y::a >= 0 ? sV[(Y::a >= 0 ? Y::a : 0) * L + i] : 0.0;
  q.b = Y::b >= 0 ? sV[(Y::b >= 0 ? Y::b : 0) * L + i] : 0.0;
  return q;
}

// Whether a stage update stores only V5 of the entropy variables: the central fluxes
// read no other, and an inviscid run forms no gradients inside its steps.  Strong
// conditions keep all four: they reset P after the update and leave the entropy
// variables of the reset vertices as the update formed them, as the reference does.
template <int FLUX>
__device__ __forceinline__ bool w3_only(const Params& k) {
  return FLUX != FLUX_TECNO_ROE && FLUX != FLUX_TECNO_RUSANOV && k.model == 0 && !k.strong;
}

template <int FLUX, int RECON, int MODE, bool ORD = false>
__global__ void __launch_bounds__(kTileThreads, (FLUX == FLUX_TECNO_ROE || FLUX == FLUX_TECNO_RUSANOV)
                                                    ? TG_FLUX_MINB : TG_FLUX_MINB_CENTRAL)
    k_tile_flux(Params k, MeshView m, TileView t, StateView s, Control ctl, Scalars* sc, int r, int do_norm,
                double* __restrict__ Pout, double* __restrict__ Wout, int lmax, int emax,
                const int* __restrict__ done) {
  if (*done) return;
  extern __shared__ double sm[];
  typedef VLayout<FLUX> Y;
  const int tile = tile_of_block<ORD>(t);
  const int l0 = t.loff[tile], L = t.loff[tile + 1] - l0;
  const int e0 = t.eoff[tile], NE = t.eoff[tile + 1] - e0;
  const int vb = t.vbeg[tile], nown = t.vbeg[tile + 1] - vb;
  const int nv = m.nv;
  constexpr bool kGrad = flux_needs_grad<FLUX, RECON>();
  double* sV = sm;                                          // Y::n * L
  double* sG = sm + Y::n * lmax;                            // 8 * L (gradient fluxes only)
  double* sX = sG + 8 * lmax;                               // 2 * L
  double* sE = sm + flux_vertex_doubles<FLUX, RECON>() * lmax;   // 4 * NE: ux uy ar ab -> fluxes
  constexpr bool kRoe = (FLUX == FLUX_TECNO_ROE);
  int* sS = reinterpret_cast<int*>(sE + 4 * emax);                 // Liou switch of the local vertices (Roe)
  int* sO = sS + (kRoe ? lmax : 0);
  unsigned int* sC = reinterpret_cast<unsigned int*>(sO + kTileThreads + 2);

  // ---- stage: vertex gathers, edge arrays, gather lists (all in flight at once)
  for (int i = threadIdx.x; i < L; i += blockDim.x) {
    int g = t.lv[l0 + i];
    cp_async8(sV + Y::Ru * L + i, s.P + (size_t)nv + g);
    cp_async8(sV + Y::Rv * L + i, s.P + (size_t)2 * nv + g);
    cp_async8(sV + Y::Rp * L + i, s.P + (size_t)3 * nv + g);
    cp_async8(sV + Y::RW3 * L + i, s.W + (size_t)3 * nv + g);
    if (Y::RW0 >= 0) cp_async8(sV + (Y::RW0 >= 0 ? Y::RW0 : 0) * L + i, s.W + g);
    if (Y::RT >= 0) cp_async8(sV + (Y::RT >= 0 ? Y::RT : 0) * L + i, s.P + g);
    if (kGrad) {
#pragma unroll
      for (int c = 0; c < 8; ++c) cp_async8(sG + c * L + i, s.G + (size_t)c * nv + g);
      cp_async8(sX + i, t.x + g);
      cp_async8(sX + L + i, t.y + g);
    }
    if (kRoe) {
      if (k.liou) cp_async4(sS + i, s.ssw + g);
      else sS[i] = 0;
    }
  }
  for (int le = threadIdx.x; le < NE; le += blockDim.x) {
    cp_async8(sE + le, t.ux + e0 + le);
    cp_async8(sE + NE + le, t.uy + e0 + le);
    cp_async8(sE + 2 * NE + le, t.ar + e0 + le);
    cp_async4(sE + 3 * NE + le, t.ab + e0 + le);
  }
  const int cbase = stage_lists(t, vb, nown, sC, sO);
  cp_async_wait_all();
  __syncthreads();

  // ---- per-vertex records, in place
  for (int i = threadIdx.x; i < L; i += blockDim.x) {
    double u = sV[Y::Ru * L + i], v = sV[Y::Rv * L + i], p = sV[Y::Rp * L + i], w3 = sV[Y::RW3 * L + i];
    double w0 = Y::RW0 >= 0 ? sV[(Y::RW0 >= 0 ? Y::RW0 : 0) * L + i] : 0.0;
    double T = Y::RT >= 0 ? sV[(Y::RT >= 0 ? Y::RT : 0) * L + i] : 0.0;
    const int g = k.strong ? t.lv[l0 + i] : 0;
    if (k.strong && (m.sflag[g] & 1)) {
      // a strong condition reset this vertex's primitive state but not its entropy
      // variables: the flux reads the primitive state, as the reference does
      Prim q;
      q.T = Y::RT >= 0 ? T : s.P[g]; q.u = u; q.v = v; q.p = p;
      store_vrec<FLUX>(sV, L, i, make_vrec<FLUX>(k, q));
    } else {
      store_vrec<FLUX>(sV, L, i, make_vrec_w<FLUX>(k, u, v, p, T, w0, w3));
    }
  }
  __syncthreads();

  // ---- edge fluxes; each result overwrites its edge's geometry slots
  for (int le = threadIdx.x; le < NE; le += blockDim.x) {
    double unx = sE[le], uny = sE[NE + le], area = sE[2 * NE + le];
    unsigned int ab = *reinterpret_cast<const unsigned int*>(sE + 3 * NE + le);
    int la = ab & 0xffff, lb = ab >> 16;
    VRec A = load_vrec<FLUX>(sV, L, la), B = load_vrec<FLUX>(sV, L, lb);
    double gl[8], gr[8], dx = 0.0, dy = 0.0;
    if (kGrad) {
#pragma unroll
      for (int c = 0; c < 8; ++c) { gl[c] = sG[c * L + la]; gr[c] = sG[c * L + lb]; }
      dx = sX[lb] - sX[la];
      dy = sX[L + lb] - sX[L + la];
    }
    Flx F = num_flux_unit<FLUX, RECON>(k, A, B, unx, uny, area, dx, dy, gl, gr, kRoe ? sS[la] + sS[lb] : 0);
    if (k.axi) {   // residual[cl] += flux * r_f, residual[cr] -= flux * r_f (src/fv.cc:1095-1096)
      const double rf = t.r[e0 + le];
      F.m *= rf; F.x *= rf; F.y *= rf; F.e *= rf;
    }
    sE[le] = F.m; sE[NE + le] = F.x; sE[2 * NE + le] = F.y; sE[3 * NE + le] = F.e;
  }
  __syncthreads();

  // ---- owned vertices: fixed-order sum, then residual or RK update
  const int tid = threadIdx.x;
  const int v = vb + tid;
  double nrm[4] = {0.0, 0.0, 0.0, 0.0};
  // last stage with fuse_dt: the next step's local dt and U_old from the new state
  const bool next_dt = MODE == MODE_UPDATE && do_norm && k.fuse_dt;
  unsigned long long dbits = 0x7ff0000000000000ull;
  Prim qn;                                   // the owned vertex's new state (next_dt)
  if (tid < nown) {
    Prim q0;
    double uo[4], area = 0.0, w = 0.0, dtl = 0.0;
    if (MODE == MODE_UPDATE) {   // issue the update's loads before the gather
      q0 = load_prim(s.P, nv, v);
#pragma unroll
      for (int c = 0; c < 4; ++c) uo[c] = s.Uold[(size_t)c * nv + v];
      area = m.dcarea[v];
      w = m.pweight[v];
      if (!(ctl.time_mode == 1 || ctl.time_step > 0.0)) dtl = s.dt[v];
    }
    double r0 = 0.0, r1 = 0.0, r2 = 0.0, r3 = 0.0;
    const int j0 = sO[tid] - cbase, j1 = sO[tid + 1] - cbase;
    for (int j = j0; j < j1; ++j) {
      int ent = list_entry(sC, j);
      int le = ent >> 1;
      double sg = (ent & 1) ? -1.0 : 1.0;
      r0 += sE[le] * sg; r1 += sE[NE + le] * sg; r2 += sE[2 * NE + le] * sg; r3 += sE[3 * NE + le] * sg;
    }
    const int n2 = 2 * m.nb, n3 = 3 * m.nvu;
    for (int j = m.cb_off[v]; j < m.cb_off[v + 1]; ++j) {
      int ent = m.cb_ent[j];
      int type = ent & 3, idx = ent >> 2;
      // axisymmetric weights (src/fv.cc:1151, 1187, 1226-1228, 1280-1282, 1315-1316): half the
      // radius of the boundary-face vertex, of the viscous unit's cell, of the vertex
      if (type == 0) {
        const double w = k.axi ? 0.5 * m.v_r[(idx & 1) ? m.b_v1[idx >> 1] : m.b_v0[idx >> 1]] : 0.5;
        r0 += s.Fb[idx] * w; r1 += s.Fb[n2 + idx] * w; r2 += s.Fb[2 * n2 + idx] * w; r3 += s.Fb[3 * n2 + idx] * w;
      } else if (type == 2 && k.model == 1) {
        const double w = k.axi ? -(0.5 * m.u_r[idx / 3]) : -(0.5 * 1.0);
        r1 += s.Fv[idx] * w; r2 += s.Fv[n3 + idx] * w; r3 += s.Fv[2 * n3 + idx] * w;
      } else if (type == 3 && k.model == 1) {
        const double w = k.axi ? 0.5 * m.v_r[v] : 0.5;
        r1 += s.Fvb[idx] * w; r2 += s.Fvb[m.nb + idx] * w; r3 += s.Fvb[2 * m.nb + idx] * w;
      }
    }
    // strong conditions: compute_residual_norm zeroes the no-slip momentum residual
    // before the last stage's update (src/fv.cc:1805-1819)
    if (MODE == MODE_UPDATE && do_norm && k.strong && (m.sflag[v] & 2)) { r1 = 0.0; r2 = 0.0; }
    if (MODE == MODE_RESIDUAL) {
      s.R[v] = r0; s.R[nv + v] = r1; s.R[2 * nv + v] = r2; s.R[3 * nv + v] = r3;
    } else {
      if (do_norm) {
        double a0 = r0 / area, a1 = r1 / area, a2 = r2 / area, a3 = r3 / area;
        nrm[0] = a0 * a0 * w; nrm[1] = a1 * a1 * w; nrm[2] = a2 * a2 * w; nrm[3] = a3 * a3 * w;
      }
      double dtv = (ctl.time_mode == 1 || ctl.time_step > 0.0) ? sc->dt_global : dtl;
      double factor = dtv / (vertex_radius(k, m, v) * area);
      Cons c = rk_stage(k, ctl, s, nv, v, r, q0, uo, factor, r0, r1, r2, r3);
      Prim q = con2prim(k, c);
      Pout[v] = q.T; Pout[nv + v] = q.u; Pout[2 * nv + v] = q.v; Pout[3 * nv + v] = q.p;
      if (w3_only<FLUX>(k)) {
        // inviscid central fluxes read only V5 = -2 beta: the other entropy variables
        // (two logarithms) are formed from P by whatever later needs them (refresh_w)
        Wout[3 * nv + v] = prim2ent_v5(k, q);
      } else {
        Ent e = prim2ent(k, q);
        Wout[v] = e.f; Wout[nv + v] = e.vx; Wout[2 * nv + v] = e.vy; Wout[3 * nv + v] = e.l;
      }
      bool ok = isfinite(q.T) && isfinite(q.u) && isfinite(q.v) && isfinite(q.p) && q.p > 0.0 && c.r > 0.0;
      if (!ok) atomicOr(&sc->bad, 1);
      if (next_dt) qn = q;
    }
  }
  if (next_dt) {
    // compute_dt (src/fv.cc:1499-1598) and store_conserved_old (src/fv.cc:1626-1630) of
    // the coming step, with the operands and order of k_tile_grad<true, *>: the tile's
    // dual normals are staged over the consumed fluxes in one wave of copies
    __syncthreads();
    for (int le = threadIdx.x; le < NE; le += blockDim.x) {
      cp_async8(sE + le, t.nx + e0 + le);
      cp_async8(sE + NE + le, t.ny + e0 + le);
    }
    cp_async_wait_all();
    __syncthreads();
    if (tid < nown) {
      const double cs = sound_speed(k, qn);
      const int j0 = sO[tid] - cbase, j1 = sO[tid + 1] - cbase;
      double lam = 0.0;
      for (int j = j0; j < j1; ++j) {
        const int le = list_entry(sC, j) >> 1;
        const double nx = sE[le], ny = sE[NE + le];
        const double ar = face_area(nx, ny);
        lam += face_radius(qn.u, qn.v, nx, ny, cs, ar) * 1.0;
      }
      for (int j = m.cb_off[v]; j < m.cb_off[v + 1]; ++j) {
        const int ent = m.cb_ent[j];
        if ((ent & 3) != 0) continue;
        const int d = ent >> 3;
        const double nx = m.b_nx[d], ny = m.b_ny[d];
        const double ar = face_area(nx, ny);
        lam += 0.5 * face_radius(qn.u, qn.v, nx, ny, cs, ar);
      }
      if (k.model == 1) {
        for (int j = j0; j < j1; ++j) {
          const int le = list_entry(sC, j) >> 1;
          const unsigned int ab = t.ab[e0 + le];
          const int ga = t.lv[l0 + (int)(ab & 0xffff)], gb = t.lv[l0 + (int)(ab >> 16)];
          const double nx = sE[le], ny = sE[NE + le];
          const double ar = face_area(nx, ny);
          const double dx = t.x[gb] - t.x[ga], dy = t.y[gb] - t.y[ga];
          const double dl = face_area(dx, dy);
          lam += (viscosity(k, qn.T) * ar / dl / density(k, qn)) * 1.0;
        }
      }
      const double dtn = k.cfl * m.dcarea[v] / lam;
      s.dt[v] = dtn;
      dbits = (unsigned long long)__double_as_longlong(dtn);
      if (!(dtn > 0.0)) dbits = 0x7ff0000000000000ull;
      const Cons un = prim2con(k, qn);
      s.Uold[v] = un.r; s.Uold[nv + v] = un.mx; s.Uold[2 * nv + v] = un.my; s.Uold[3 * nv + v] = un.E;
    }
    dbits = block_min_u64(dbits);
    if (threadIdx.x == 0) {
      atomicMin(&sc->dtmin_next, dbits);
      if (blockIdx.x == 0) sc->dt_next = 1;
    }
  }
  if (MODE == MODE_UPDATE && do_norm) {
    // the tile buffers are no longer needed: reuse them for the block reduction
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
      for (int c = 0; c < 4; ++c) s.part[(size_t)((ORD ? t.base : 0) + blockIdx.x) * 4 + c] = red[c * kTileThreads];
    // the last block to finish forms the norms and ends the step
    __shared__ int last;
    if (threadIdx.x == 0) {
      __threadfence();
      last = atomicAdd(&sc->blocks_done, 1u) == (ORD ? (unsigned)t.total : gridDim.x) - 1;
    }
    __syncthreads();
    if (last) {
      __threadfence();
      norm_and_step_end(s, ORD ? t.total : (int)gridDim.x, nv, sc, ctl, red, kTileThreads);
      if (threadIdx.x == 0) sc->blocks_done = 0;
    }
  }
}

// gather-list words (cmax entries, two per word) + offsets
inline size_t tile_list_bytes(int cmax) {
  return (kTileThreads + 2) * sizeof(int) + (size_t)((cmax + 2) / 2 + 1) * sizeof(unsigned int);
}

inline size_t tile_grad_smem(int lmax, int emax, int cmax, bool first) {
  return ((size_t)lmax * grad_vertex_doubles(first) + (size_t)emax * grad_edge_doubles(first)) * sizeof(double) +
         (size_t)emax * sizeof(unsigned int) + tile_list_bytes(cmax);
}

template <int FLUX, int RECON>
size_t tile_flux_smem_t(int lmax, int emax, int cmax) {
  size_t a = ((size_t)lmax * flux_vertex_doubles<FLUX, RECON>() + 4 * (size_t)emax) * sizeof(double) +
             (FLUX == FLUX_TECNO_ROE ? (size_t)lmax * sizeof(int) : 0) + tile_list_bytes(cmax);
  size_t b = 4 * kTileThreads * sizeof(double);
  return a > b ? a : b;
}

}  // namespace tg
