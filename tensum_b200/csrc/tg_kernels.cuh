// tg_kernels.cuh -- device kernels of the FP64 single-solve path.
//
// One launch per reference phase; every accumulation is a fixed-order gather
// over per-vertex lists built on the host (tg_mesh.cc), so results are
// bitwise reproducible from run to run.
#pragma once

#include <cstdint>

#include "tg_physics.cuh"

namespace tg {

constexpr int kBlock = 256;

struct MeshView {
  int nv, ne, nb, nvu, n_int_cells;
  const double *dcarea, *inv6mc, *pweight;
  const int *e_a, *e_b;
  const double *e_nx, *e_ny, *e_dx, *e_dy, *e_g0x, *e_g0y, *e_g1x, *e_g1y;
  const int *ce_off, *ce_ent;
  const int *cb_off, *cb_ent;
  const int *b_v0, *b_v1, *b_kind, *b_adiab, *b_cell;
  const double *b_nx, *b_ny, *b_val;
  const double *bf_face_nx, *bf_face_ny;
  const int *bf_face_v0, *bf_face_v1;
  const int* u_cell;
  const int* c_v;
  const double *c_n, *c_inv2a;
  const int *c_bf_off, *c_bf, *c_nbr_off, *c_nbr;
  // bc_scheme strong: per vertex bit 0 = a boundary condition resets its state,
  // bit 1 = on a no-slip face; the reset list (vertex, then (face << 1 | slot)
  // entries in reference face order)
  const int* sflag;
  int nsb;
  const int *sb_v, *sb_off, *sb_ent;
  // axisymmetric radii (src/grid_preproc.cc:750-777): per vertex and per viscous unit
  const double *v_r, *u_r;
};

// Vertex radius of an axisymmetric run (1 when planar): update_solution divides
// by radius x dual area (src/fv.cc:1646, 1671, 1685).
__device__ __forceinline__ double vertex_radius(const Params& k, const MeshView& m, int v) {
  return k.axi ? m.v_r[v] : 1.0;
}

// Device state, structure-of-arrays with component stride nv (or ne, nb ...).
struct StateView {
  double* P;      // 4*nv  T,u,v,p
  double* W;      // 4*nv  V1,V2,V3,V5
  double* G;      // 8*nv  dV1/dx, dV1/dy, dV2/dx, ..., dV5/dy
  double* R;      // 4*nv
  double* Uold;   // 4*nv
  double* dt;     // nv
  double* Fe;     // 4*ne
  double* Fb;     // 4*2*nb
  double* Fv;     // 3*3*nvu  (x-mom, y-mom, energy)
  double* Fvb;    // 3*nb
  double* part;   // block partial sums
  double* R2;     // 4*nv  RK4 residual accumulator (residual2 of src/fv.h)
  int* ssw;       // nv    Liou shock switch (src/fv.h:160)
};

// Step bookkeeping kept on the device so that whole steps replay from a CUDA graph.
struct Scalars {
  double dt_global;
  double elapsed;
  double rtotal;
  double rtotal0;
  double rnorm[4];
  long long iter;
  int counter;
  int reached;
  int done;
  int bad;
  unsigned long long dtmin_bits;
  int stop_counter;    // steps stop once counter exceeds it (output-time stepping)
  // Set by a last-stage update that also formed dt, U_old and their minimum
  // (dtmin_next) for the state it wrote; cleared whenever the state changes by
  // any other route, so the next step's first stage then forms them itself.
  int dt_next;
  unsigned long long dtmin_next;
  unsigned int blocks_done;   // blocks of the last stage's launch that have written their norm partials
  double rsq[4];              // a partition's residual-norm sums of its last step, before the exchange
};

struct Control {
  int time_mode;       // 0 steady, 1 unsteady
  int n_rks;           // stages per step: 3 (ssprk3) or 4 (rk4)
  int scheme;          // 0 ssprk3, 1 rk4
  int ntinst;
  double time_step;
  double min_residue;
  long long max_iter;
  double final_time;
  const double* tinst;
  int part;            // a partition of a decomposed mesh: norms wait for the other partitions' sums
};

__device__ __forceinline__ Prim load_prim(const double* P, int nv, int i) {
  Prim q;
  q.T = P[i]; q.u = P[nv + i]; q.v = P[2 * nv + i]; q.p = P[3 * nv + i];
  return q;
}

// Boundary correction n_b * (W_b0 + W_b1 - W_0 - W_1)/2 of one boundary face
// (src/fv.cc:926-966): states after the single-state BC at each face vertex.
__device__ __forceinline__ void bface_grad_corr(const Params& k, const MeshView& m, const StateView& s, int d,
                                                double* dW /*4*/) {
  int v0 = m.b_v0[d], v1 = m.b_v1[d];
  Prim s0 = load_prim(s.P, m.nv, v0), s1 = load_prim(s.P, m.nv, v1);
  double nx = m.b_nx[d], ny = m.b_ny[d];
  bc_apply1(m.b_kind[d], m.b_adiab[d], m.b_val + (size_t)d * 10, nx, ny, s0);
  bc_apply1(m.b_kind[d], m.b_adiab[d], m.b_val + (size_t)d * 10 + 5, nx, ny, s1);
  Ent e0 = prim2ent(k, s0), e1 = prim2ent(k, s1);
  const double* W = s.W;
  const int nv = m.nv;
  dW[0] = (e0.f + e1.f - W[v0] - W[v1]) / 2.0;
  dW[1] = (e0.vx + e1.vx - W[nv + v0] - W[nv + v1]) / 2.0;
  dW[2] = (e0.vy + e1.vy - W[2 * nv + v0] - W[2 * nv + v1]) / 2.0;
  dW[3] = (e0.l + e1.l - W[3 * nv + v0] - W[3 * nv + v1]) / 2.0;
}

// ------------------------------------------------------------------ kernels

__global__ void k_prim2ent(Params k, int nv, const double* __restrict__ P, double* __restrict__ W) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  Ent e = prim2ent(k, load_prim(P, nv, i));
  W[i] = e.f; W[nv + i] = e.vx; W[2 * nv + i] = e.vy; W[3 * nv + i] = e.l;
}

// A caller state arrives as PrimVar records (T, p, u, v, w; src/primvar.h:17-18) in the caller's
// vertex order.  k_state_check flags any vertex the reference would refuse at
// initialisation (src/fv.cc:388-389: T > 0 and p > 0, NaN refused too);
// k_state_in then reorders into the device SoA only when nothing was flagged,
// so a refused state leaves the previous one in place.
__global__ void k_state_check(int nv, const double* __restrict__ raw, int* __restrict__ bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  const double* q = raw + 5 * (size_t)i;
  if (!(q[0] > 0.0) || !(q[1] > 0.0)) atomicOr(bad, 1);
}

__global__ void k_state_in(int nv, const double* __restrict__ raw, const int* __restrict__ old_of_new,
                           const int* __restrict__ bad, double* __restrict__ P) {
  if (*bad) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  const double* q = raw + 5 * (size_t)old_of_new[i];
  P[i] = q[0]; P[nv + i] = q[2]; P[2 * (size_t)nv + i] = q[3]; P[3 * (size_t)nv + i] = q[1];
}

// Device SoA (T, u, v, p) -> PrimVar records in the caller's order (w = 0 in 2D).
__global__ void k_state_out(int nv, const double* __restrict__ P, const int* __restrict__ old_of_new,
                            double* __restrict__ raw) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  double* q = raw + 5 * (size_t)old_of_new[i];
  q[0] = P[i]; q[1] = P[3 * (size_t)nv + i]; q[2] = P[nv + i]; q[3] = P[2 * (size_t)nv + i]; q[4] = 0.0;
}

// A state handed in asynchronously (tg_set_state_async) becomes current only if
// k_state_check accepted it: its entropy variables and fresh step bookkeeping.
__global__ void k_prim2ent_checked(Params k, int nv, const double* __restrict__ P, double* __restrict__ W,
                                   const int* __restrict__ bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv || *bad) return;
  Ent e = prim2ent(k, load_prim(P, nv, i));
  W[i] = e.f; W[nv + i] = e.vx; W[2 * nv + i] = e.vy; W[3 * nv + i] = e.l;
}

__global__ void k_scalars_set(Scalars* sc, Scalars s0, const int* __restrict__ bad) {
  if (*bad) return;
  *sc = s0;
}

// Device gradients G (V1, V2, V3, V5) x (x, y) -> the reference's dE records,
// 5 variables x (x, y, z) per vertex in the caller's order (src/fv.h:148),
// zero for the z components and for the fourth (z-momentum) variable.
// zero_unstepped: all zero while no step has run since the state was set (the
// reference zeroes dE when a sample starts, src/fv.cc:207-212).
__global__ void k_grad_out(int nv, const double* __restrict__ G, const int* __restrict__ old_of_new,
                           double* __restrict__ out, const Scalars* __restrict__ sc, int zero_unstepped) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  double* d = out + 15 * (size_t)old_of_new[i];
  const int var_of[4] = {0, 1, 2, 4};
#pragma unroll
  for (int q = 0; q < 15; ++q) d[q] = 0.0;
  if (zero_unstepped && sc->iter == 0) return;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    d[3 * var_of[c]] = G[(size_t)(2 * c) * nv + i];
    d[3 * var_of[c] + 1] = G[(size_t)(2 * c + 1) * nv + i];
  }
}

// store_conserved_old (src/fv.cc:1626-1630)
__global__ void k_store_old(Params k, MeshView m, StateView s, const int* __restrict__ done) {
  if (*done) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nv) return;
  Cons c = prim2con(k, load_prim(s.P, m.nv, i));
  s.Uold[i] = c.r; s.Uold[m.nv + i] = c.mx; s.Uold[2 * m.nv + i] = c.my; s.Uold[3 * m.nv + i] = c.E;
}

// Boundary-face inviscid fluxes (src/fv.cc:1100-1188): one thread per (face, vertex).
template <int FLUX, int RECON>
__global__ void k_bflux(Params k, MeshView m, StateView s, const int* __restrict__ done) {
  if (*done) return;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * m.nb) return;
  int d = t >> 1, q = t & 1;
  int c = q ? m.b_v1[d] : m.b_v0[d];
  Prim s0 = load_prim(s.P, m.nv, c), s1 = s0;
  double nx = m.b_nx[d], ny = m.b_ny[d];
  int kind = m.b_kind[d];
  bc_apply2(kind, m.b_adiab[d], m.b_val + (size_t)d * 10 + 5 * q, nx, ny, s0, s1);
  Flx F;
  if (kind == BC_FARFIELD) {
    double z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    F = num_flux<FLUX, RECON>(k, make_vrec<FLUX>(k, s0), make_vrec<FLUX>(k, s1), nx, ny, 0.0, 0.0, z, z);
  } else {
    F = inviscid_bflux(k, s0, s1, nx, ny);
  }
  const int n2 = 2 * m.nb;
  s.Fb[t] = F.m; s.Fb[n2 + t] = F.x; s.Fb[2 * n2 + t] = F.y; s.Fb[3 * n2 + t] = F.e;
}

// Viscous residual units (src/fv.cc:1197-1320): interior cells and boundary faces.
__global__ void k_viscous(Params k, MeshView m, StateView s, const int* __restrict__ done) {
  if (*done) return;
  int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= m.nvu) return;
  const int nv = m.nv;
  int c = m.u_cell[u];
  int v[3] = {m.c_v[3 * c], m.c_v[3 * c + 1], m.c_v[3 * c + 2]};
  const double* n = m.c_n + 6 * (size_t)c;
  // cell gradient: P1 sum, boundary corrections in face order, / (2 area)
  double dE[8];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double w0 = s.W[q * nv + v[0]], w1 = s.W[q * nv + v[1]], w2 = s.W[q * nv + v[2]];
    dE[2 * q] = n[0] * w0 + n[2] * w1 + n[4] * w2;
    dE[2 * q + 1] = n[1] * w0 + n[3] * w1 + n[5] * w2;
  }
  for (int j = m.c_bf_off[c]; j < m.c_bf_off[c + 1]; ++j) {
    int d = m.c_bf[j];
    double dW[4];
    bface_grad_corr(k, m, s, d, dW);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      dE[2 * q] += m.b_nx[d] * dW[q];
      dE[2 * q + 1] += m.b_ny[d] * dW[q];
    }
  }
  double f = m.c_inv2a[c];
#pragma unroll
  for (int q = 0; q < 8; ++q) dE[q] *= f;

  Ent avg;
  if (u < m.n_int_cells) {
    const double t3 = 1.0 / 3.0;
    avg.f = s.W[v[0]] * t3 + s.W[v[1]] * t3 + s.W[v[2]] * t3;
    avg.vx = s.W[nv + v[0]] * t3 + s.W[nv + v[1]] * t3 + s.W[nv + v[2]] * t3;
    avg.vy = s.W[2 * nv + v[0]] * t3 + s.W[2 * nv + v[1]] * t3 + s.W[2 * nv + v[2]] * t3;
    avg.l = s.W[3 * nv + v[0]] * t3 + s.W[3 * nv + v[1]] * t3 + s.W[3 * nv + v[2]] * t3;
  } else {
    avg.f = avg.vx = avg.vy = avg.l = 0.0;
    int cnt = m.c_nbr_off[c + 1] - m.c_nbr_off[c];
    for (int j = m.c_nbr_off[c]; j < m.c_nbr_off[c + 1]; ++j) {
      int d = m.c_nbr[j];
      for (int q = 0; q < 2; ++q) {
        int vb = q ? m.bf_face_v1[d] : m.bf_face_v0[d];
        Prim st = load_prim(s.P, nv, vb);
        const double* val = m.b_val + (size_t)d * 10 + (vb == m.b_v0[d] ? 0 : 5);
        bc_apply1(m.b_kind[d], m.b_adiab[d], val, m.bf_face_nx[d], m.bf_face_ny[d], st);
        Ent e = prim2ent(k, st);
        avg.f += e.f; avg.vx += e.vx; avg.vy += e.vy; avg.l += e.l;
      }
    }
    double sc = (0.5 * 1.0 / cnt);
    avg.f *= sc; avg.vx *= sc; avg.vy *= sc; avg.l *= sc;
  }
  ViscK K = viscous_K(k, avg, dE);
  const int n3 = 3 * m.nvu;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    Flx F = viscous_apply(K, n[2 * q], n[2 * q + 1]);
    s.Fv[3 * u + q] = F.x; s.Fv[n3 + 3 * u + q] = F.y; s.Fv[2 * n3 + 3 * u + q] = F.e;
  }
  if (u >= m.n_int_cells) {
    int d = u - m.n_int_cells;
    double nbx = m.b_nx[d], nby = m.b_ny[d];
    double Cor = m.b_adiab[d] ? -1.0 * (0.0 + K.c2 * K.e4 * K.e4 * (dE[6] * nbx + dE[7] * nby)) : 0.0;
    Flx F = viscous_apply(K, nbx, nby);
    s.Fvb[d] = F.x; s.Fvb[m.nb + d] = F.y; s.Fvb[2 * m.nb + d] = F.e - Cor;
  }
}

// |n| and the face spectral radius |u.n| + c |n| of the local time step
// (src/fv.cc:1512-1580), with their multiply-adds written out so that every
// kernel forming them rounds them the same way.
__device__ __forceinline__ double face_area(double nx, double ny) { return sqrt(fma(nx, nx, ny * ny)); }
__device__ __forceinline__ double face_radius(double u, double v, double nx, double ny, double c, double area) {
  return fma(c, area, fabs(fma(u, nx, v * ny)));
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long y = __shfl_xor_sync(0xffffffffu, x, o);
    x = y < x ? y : x;
  }
  return x;
}

// Local time step (src/fv.cc:1499-1598): spectral-radius gather, dt = cfl A / sum,
// block minimum by warp shuffles, then one atomicMin on the (positive) bit pattern.
__global__ void k_dt(Params k, MeshView m, StateView s, Scalars* sc, const int* __restrict__ done) {
  if (*done) return;
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long bits = 0x7ff0000000000000ull;  // +inf
  if (v < m.nv) {
    const int nv = m.nv;
    double lam = 0.0;
    for (int j = m.ce_off[v]; j < m.ce_off[v + 1]; ++j) {
      int ent = m.ce_ent[j];
      int e = ent >> 1;
      int self = (ent & 1) ? m.e_b[e] : m.e_a[e];
      Prim q = load_prim(s.P, nv, self);
      double nx = m.e_nx[e], ny = m.e_ny[e];
      double area = face_area(nx, ny);
      lam += face_radius(q.u, q.v, nx, ny, sound_speed(k, q), area) * 1.0;
    }
    for (int j = m.cb_off[v]; j < m.cb_off[v + 1]; ++j) {
      int ent = m.cb_ent[j];
      if ((ent & 3) != 0) continue;
      int idx = ent >> 2, d = idx >> 1;
      int self = (idx & 1) ? m.b_v1[d] : m.b_v0[d];
      Prim q = load_prim(s.P, nv, self);
      double nx = m.b_nx[d], ny = m.b_ny[d];
      double area = face_area(nx, ny);
      lam += 0.5 * face_radius(q.u, q.v, nx, ny, sound_speed(k, q), area);
    }
    if (k.model == 1) {
      for (int j = m.ce_off[v]; j < m.ce_off[v + 1]; ++j) {
        int ent = m.ce_ent[j];
        int e = ent >> 1;
        int self = (ent & 1) ? m.e_b[e] : m.e_a[e];
        Prim q = load_prim(s.P, nv, self);
        double nx = m.e_nx[e], ny = m.e_ny[e];
        double area = face_area(nx, ny);
        double dl = face_area(m.e_dx[e], m.e_dy[e]);
        lam += (viscosity(k, q.T) * area / dl / density(k, q)) * 1.0;
      }
    }
    double dtv = k.cfl * m.dcarea[v] / lam;
    s.dt[v] = dtv;
    bits = (unsigned long long)__double_as_longlong(dtv);
    if (!(dtv > 0.0)) bits = 0x7ff0000000000000ull;  // NaN / non-positive: flagged by the update
  }
  bits = warp_min_u64(bits);
  __shared__ unsigned long long wmin[kBlock / 32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) wmin[w] = bits;
  __syncthreads();
  if (w == 0) {
    bits = lane < (int)(blockDim.x >> 5) ? wmin[lane] : 0x7ff0000000000000ull;
    bits = warp_min_u64(bits);
    if (lane == 0) atomicMin(&sc->dtmin_bits, bits);
  }
}

// Start of a solve-loop iteration (src/fv.cc:2273-2276): loop condition and dt reset.
// compute_ssw (src/compute_ssw.cc:7-38): flags both endpoints of every edge
// (all faces, boundary ones included) across which u.n - a|n| or u.n + a|n|
// changes sign from positive to negative.  Writers only ever store 1.
__global__ void k_ssw(Params k, MeshView m, StateView s, const int* __restrict__ done) {
  if (*done) return;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m.ne) return;
  const int a = m.e_a[e], b = m.e_b[e];
  const Prim qa = load_prim(s.P, m.nv, a), qb = load_prim(s.P, m.nv, b);
  const double nx = m.e_nx[e], ny = m.e_ny[e];
  const double ui = qa.u * nx + qa.v * ny, uj = qb.u * nx + qb.v * ny;
  const double ai = sound_speed(k, qa), aj = sound_speed(k, qb);
  const double area = sqrt(nx * nx + ny * ny);
  const double l1i = ui - ai * area, l1j = uj - aj * area;
  const double l5i = ui + ai * area, l5j = uj + aj * area;
  if ((l1i > 0 && l1j < 0) || (l5i > 0 && l5j < 0)) {
    s.ssw[a] = 1;
    s.ssw[b] = 1;
  }
}

// bc_scheme strong, after each stage update (src/fv.cc:1694-1704): every
// boundary face's condition applied to its vertices' primitive state in face
// order; the entropy variables keep their values (the reference does not
// recompute them), so gradients see the pre-condition state.
__global__ void k_strong_bc(MeshView m, double* __restrict__ P, const int* __restrict__ done) {
  if (*done) return;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m.nsb) return;
  const int v = m.sb_v[j], nv = m.nv;
  Prim q = load_prim(P, nv, v);
  for (int e = m.sb_off[j]; e < m.sb_off[j + 1]; ++e) {
    const int d = m.sb_ent[e] >> 1, slot = m.sb_ent[e] & 1;
    bc_apply1(m.b_kind[d], m.b_adiab[d], m.b_val + (size_t)d * 10 + 5 * slot, m.b_nx[d], m.b_ny[d], q);
  }
  P[v] = q.T; P[nv + v] = q.u; P[2 * (size_t)nv + v] = q.v; P[3 * (size_t)nv + v] = q.p;
}

// bc_scheme strong, in compute_residual_norm (src/fv.cc:1805-1819): the momentum
// residual of no-slip vertices is zeroed (the update then uses it).
__global__ void k_strong_zero_res(MeshView m, StateView s) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= m.nv || !(m.sflag[v] & 2)) return;
  s.R[m.nv + v] = 0.0;
  s.R[2 * (size_t)m.nv + v] = 0.0;
}

// Global dt and the unsteady clamp to the next output time (src/fv.cc:1584-1618).
__device__ __forceinline__ void dt_final(const Control& ctl, Scalars* sc) {
  double dtg;
  if (ctl.time_step > 0.0) {
    dtg = ctl.time_step;
  } else {
    dtg = 1.0e20;
    double m = __longlong_as_double((long long)sc->dtmin_bits);
    dtg = dmin_(dtg, m);
    if (ctl.time_mode == 1) {
      int c = sc->counter < ctl.ntinst ? sc->counter : ctl.ntinst - 1;
      if (sc->elapsed + dtg > ctl.tinst[c]) {
        dtg = ctl.tinst[c] - sc->elapsed;
        sc->reached = 1;
      }
    }
  }
  sc->dt_global = dtg;
}

__global__ void k_dt_final(Control ctl, Scalars* sc, const int* __restrict__ done) {
  if (*done) return;
  dt_final(ctl, sc);
}

// Start of a solve-loop iteration: the loop condition, and the running dt
// minimum -- the previous step's last update already formed it for this state
// when dt_next is set.  warm (a step captured without the first-stage dt pass,
// launched only when dt_next is set): the dt clamp happens here too.
__global__ void k_step_begin(Control ctl, Scalars* sc, int* done, int warm) {
  // unsteady runs never advance the iteration bound (term_iter stays 0, src/fv.cc:2266-2268)
  bool go = sc->rtotal > ctl.min_residue && (ctl.time_mode == 1 || sc->iter < ctl.max_iter) &&
            sc->elapsed < ctl.final_time && sc->counter <= sc->stop_counter;
  *done = go ? 0 : 1;
  if (!go) return;
  sc->dtmin_bits = sc->dt_next ? sc->dtmin_next : 0x7ff0000000000000ull;
  sc->dtmin_next = 0x7ff0000000000000ull;
  if (warm) dt_final(ctl, sc);
}

// Residual norms from the weighted squared sums of the whole mesh (src/fv.cc:1846-1876);
// the first iteration's total becomes the reference for the relative residual.
__device__ __forceinline__ void set_norms(Scalars* sc, const double* sum4, int nv_total, bool first) {
  double n0 = sqrt(sum4[0]) / nv_total, n1 = sqrt(sum4[1]) / nv_total;
  double n2 = sqrt(sum4[2]) / nv_total, n3 = sqrt(sum4[3]) / nv_total;
  double total = sqrt(n0 * n0 + (n1 * n1 + n2 * n2 + 0.0) + n3 * n3);
  if (first) {
    sc->rtotal0 = total;
    if (sc->rtotal0 == 0.0) sc->rtotal0 = 1.0;
  }
  sc->rnorm[0] = n0; sc->rnorm[1] = n1; sc->rnorm[2] = n2; sc->rnorm[3] = n3;
  sc->rtotal = total / sc->rtotal0;
}

// Residual norms from the per-block partials (src/fv.cc:1846-1876) and the end
// of the solve-loop iteration (src/fv.cc:2307-2343), by one block of `threads`
// threads (red: 4 * threads doubles of shared memory).
__device__ __forceinline__ void norm_and_step_end(const StateView& s, int nblocks, int nv_total, Scalars* sc,
                                                  const Control& ctl, double* red, int threads) {
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
  for (int b = threadIdx.x; b < nblocks; b += threads)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[c] += __ldcg(s.part + (size_t)b * 4 + c);
#pragma unroll
  for (int c = 0; c < 4; ++c) red[c * threads + threadIdx.x] = acc[c];
  __syncthreads();
  for (int o = threads / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
#pragma unroll
      for (int c = 0; c < 4; ++c) red[c * threads + threadIdx.x] += red[c * threads + threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double sum4[4] = {red[0], red[threads], red[2 * threads], red[3 * threads]};
    if (ctl.part) {
#pragma unroll
      for (int c = 0; c < 4; ++c) sc->rsq[c] = sum4[c];
    } else {
      set_norms(sc, sum4, nv_total, sc->iter == 0);
    }
    sc->iter += 1;
    sc->elapsed += sc->dt_global;
    if (sc->reached && ctl.time_mode == 1) {
      sc->counter += 1;
      sc->reached = 0;
    }
  }
}

// update_solution for SSP-RK3 (src/fv.cc:1641-1652), fused with the residual-norm
// partial sums of compute_residual_norm (src/fv.cc:1822-1841) at the last stage.
// New conserved state of vertex v at stage r from its residual: the Shu-Osher
// SSP-RK3 stage (src/fv.cc:1635-1658, src/constants.h:4-6) or the classical RK4
// stage (src/fv.cc:1667-1679, src/constants.h:9), which accumulates
// sum_r R_r / rks_r in R2 (zero before the first stage, src/fv.cc:2287-2293).
// q0 is the stage's input state, uo U_old, factor = dt / area.
__device__ __forceinline__ Cons rk_stage(const Params& k, const Control& ctl, const StateView& s, int nv, int v, int r,
                                         const Prim& q0, const double* uo, double factor, double r0, double r1,
                                         double r2, double r3) {
  Cons c;
  if (ctl.scheme == 1) {
    const double rks[4] = {1.0, 1.0 / 2.0, 1.0 / 2.0, 1.0};
    const double inv = 1.0 / rks[r];
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    if (r > 0) { a0 = s.R2[v]; a1 = s.R2[nv + v]; a2 = s.R2[2 * nv + v]; a3 = s.R2[3 * nv + v]; }
    a0 += r0 * inv; a1 += r1 * inv; a2 += r2 * inv; a3 += r3 * inv;
    if (r < 3) { s.R2[v] = a0; s.R2[nv + v] = a1; s.R2[2 * nv + v] = a2; s.R2[3 * nv + v] = a3; }
    const bool fin = (r == 3);
    const double c2 = fin ? -factor / 6.0 : -factor * rks[r < 3 ? r + 1 : 3];
    c.r = uo[0] * 1.0 + (fin ? a0 : r0) * c2;
    c.mx = uo[1] * 1.0 + (fin ? a1 : r1) * c2;
    c.my = uo[2] * 1.0 + (fin ? a2 : r2) * c2;
    c.E = uo[3] * 1.0 + (fin ? a3 : r3) * c2;
    return c;
  }
  const double a_rk[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0};
  const double b_rk[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
  c = prim2con(k, q0);
  const double br = b_rk[r], ar = a_rk[r], c2 = -factor * br;
  c.r *= br; c.mx *= br; c.my *= br; c.E *= br;
  c.r += uo[0] * ar + r0 * c2;
  c.mx += uo[1] * ar + r1 * c2;
  c.my += uo[2] * ar + r2 * c2;
  c.E += uo[3] * ar + r3 * c2;
  return c;
}

__global__ void k_update(Params k, MeshView m, StateView s, Control ctl, Scalars* sc, int r, int do_norm,
                         const int* __restrict__ done) {
  if (*done) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nv = m.nv;
  double nrm[4] = {0.0, 0.0, 0.0, 0.0};
  if (i < nv) {
    double R0 = s.R[i], R1 = s.R[nv + i], R2 = s.R[2 * nv + i], R3 = s.R[3 * nv + i];
    double area = m.dcarea[i];
    if (do_norm) {
      double w = m.pweight[i];
      double q0 = R0 / area, q1 = R1 / area, q2 = R2 / area, q3 = R3 / area;
      nrm[0] = q0 * q0 * w; nrm[1] = q1 * q1 * w; nrm[2] = q2 * q2 * w; nrm[3] = q3 * q3 * w;
    }
    double dtv = (ctl.time_mode == 1 || ctl.time_step > 0.0) ? sc->dt_global : s.dt[i];
    double factor = dtv / (vertex_radius(k, m, i) * area);
    const double uo[4] = {s.Uold[i], s.Uold[nv + i], s.Uold[2 * nv + i], s.Uold[3 * nv + i]};
    Cons c = rk_stage(k, ctl, s, nv, i, r, load_prim(s.P, nv, i), uo, factor, R0, R1, R2, R3);
    Prim q = con2prim(k, c);
    Ent e = prim2ent(k, q);
    s.P[i] = q.T; s.P[nv + i] = q.u; s.P[2 * nv + i] = q.v; s.P[3 * nv + i] = q.p;
    s.W[i] = e.f; s.W[nv + i] = e.vx; s.W[2 * nv + i] = e.vy; s.W[3 * nv + i] = e.l;
    bool ok = isfinite(q.T) && isfinite(q.u) && isfinite(q.v) && isfinite(q.p) && q.p > 0.0 && c.r > 0.0;
    if (!ok) atomicOr(&sc->bad, 1);
  }
  if (do_norm) {
    // fixed-shape block reduction -> per-block partials, summed in block order later
    __shared__ double red[4][kBlock];
#pragma unroll
    for (int c = 0; c < 4; ++c) red[c][threadIdx.x] = nrm[c];
    __syncthreads();
    for (int o = kBlock / 2; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o)
#pragma unroll
        for (int c = 0; c < 4; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0)
#pragma unroll
      for (int c = 0; c < 4; ++c) s.part[(size_t)blockIdx.x * 4 + c] = red[c][0];
  }
}

// Residual-norm partial sums alone (src/fv.cc:1822-1841), same reduction shape as k_update.
__global__ void k_norm_part(MeshView m, StateView s, const int* __restrict__ done) {
  if (*done) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nv = m.nv;
  double nrm[4] = {0.0, 0.0, 0.0, 0.0};
  if (i < nv) {
    double area = m.dcarea[i], w = m.pweight[i];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      double q = s.R[c * nv + i] / area;
      nrm[c] = q * q * w;
    }
  }
  __shared__ double red[4][kBlock];
#pragma unroll
  for (int c = 0; c < 4; ++c) red[c][threadIdx.x] = nrm[c];
  __syncthreads();
  for (int o = kBlock / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
#pragma unroll
      for (int c = 0; c < 4; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int c = 0; c < 4; ++c) s.part[(size_t)blockIdx.x * 4 + c] = red[c][0];
}

// Norm finalisation (src/fv.cc:1846-1876): one block sums the partials in a fixed order.
__global__ void k_norm_final(StateView s, int nblocks, int nv_total, Scalars* sc, int use_sc_iter, long long iter,
                             const int* __restrict__ done) {
  if (*done) return;
  __shared__ double red[4][kBlock];
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  // unrolled so that several partials' loads are in flight before the ordered adds
#pragma unroll 8
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[c] += s.part[(size_t)b * 4 + c];
#pragma unroll
  for (int c = 0; c < 4; ++c) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int o = kBlock / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
#pragma unroll
      for (int c = 0; c < 4; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double n0 = sqrt(red[0][0]) / nv_total, n1 = sqrt(red[1][0]) / nv_total;
    double n2 = sqrt(red[2][0]) / nv_total, n3 = sqrt(red[3][0]) / nv_total;
    double total = sqrt(n0 * n0 + (n1 * n1 + n2 * n2 + 0.0) + n3 * n3);
    long long it = use_sc_iter ? sc->iter : iter;
    if (it == 0) {
      sc->rtotal0 = total;
      if (sc->rtotal0 == 0.0) sc->rtotal0 = 1.0;
    }
    sc->rnorm[0] = n0; sc->rnorm[1] = n1; sc->rnorm[2] = n2; sc->rnorm[3] = n3;
    sc->rtotal = total / sc->rtotal0;
  }
}

// End of a solve-loop iteration (src/fv.cc:2307-2343).
__global__ void k_step_end(Control ctl, Scalars* sc, const int* __restrict__ done) {
  if (*done) return;
  sc->iter += 1;
  sc->elapsed += sc->dt_global;
  if (sc->reached && ctl.time_mode == 1) {
    sc->counter += 1;
    sc->reached = 0;
  }
}

// Kinetic-energy and entropy integrals (src/fv.cc:2186-2203), block partials.
__global__ void k_global(Params k, MeshView m, StateView s) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double ke = 0.0, en = 0.0;
  if (i < m.nv) {
    Prim q = load_prim(s.P, m.nv, i);
    double w = m.pweight[i], A = m.dcarea[i];
    double rho = density(k, q);
    ke = (0.5 * rho * (q.u * q.u + q.v * q.v) * A) * w;
    en = (-rho * entropy_fn(k, q) / (k.gamma - 1.0)) * A * w;
  }
  __shared__ double red[2][kBlock];
  red[0][threadIdx.x] = ke;
  red[1][threadIdx.x] = en;
  __syncthreads();
  for (int o = kBlock / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      red[0][threadIdx.x] += red[0][threadIdx.x + o];
      red[1][threadIdx.x] += red[1][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) { s.part[(size_t)blockIdx.x * 4] = red[0][0]; s.part[(size_t)blockIdx.x * 4 + 1] = red[1][0]; }
}

// ------------------------------------------------------------ forces
// compute_forces (src/force.cc:116-219) for the force of block f: pressure
// force sum over faces of 0.5 (p0 + p1) n and, for Navier-Stokes, the viscous
// stress from the vertex gradients of u and v recovered from those of the
// entropy variables.  Face record (d, dq, k0, k1): the face's device index, and
// -- as the reference applies the condition of bface[f] with f the force
// index -- the device index of bface[f] (-1: no condition) with the value
// slots its evaluation uses.  Fixed-order block reduction.
__global__ void k_forces(Params k, MeshView m, StateView s, const int4* __restrict__ faces,
                         const int* __restrict__ off, double* __restrict__ out) {
  const int f = blockIdx.x;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  const int nv = m.nv;
  for (int j = off[f] + threadIdx.x; j < off[f + 1]; j += blockDim.x) {
    const int4 r = faces[j];
    const int d = r.x, dq = r.y;
    const int v0 = m.b_v0[d], v1 = m.b_v1[d];
    const double nx = m.b_nx[d], ny = m.b_ny[d];
    Prim s0 = load_prim(s.P, nv, v0), s1 = load_prim(s.P, nv, v1);
    if (dq >= 0) {
      bc_apply1(m.b_kind[dq], m.b_adiab[dq], m.b_val + (size_t)dq * 10 + 5 * r.z, m.b_nx[dq], m.b_ny[dq], s0);
      bc_apply1(m.b_kind[dq], m.b_adiab[dq], m.b_val + (size_t)dq * 10 + 5 * r.w, m.b_nx[dq], m.b_ny[dq], s1);
    }
    const double pr = 0.5 * (s0.p + s1.p);
    acc[0] += nx * pr;
    acc[1] += ny * pr;
    if (k.model == 1) {
      const Ent e0 = prim2ent(k, s0), e1 = prim2ent(k, s1);
      const double T = (s0.T + s1.T) / 2.0;
      const double mu = viscosity(k, T);
      const double f0 = 1.0 / e0.l, f1 = 1.0 / e1.l;
      const double* G = s.G;
      auto g = [&](int c, int v) { return G[(size_t)c * nv + v]; };
      // u = -V2 / V5: grad u = -grad V2 / V5 + V2 grad V5 / V5^2 (src/force.cc:169-179)
      const double ux0 = g(2, v0) * -f0 + g(6, v0) * (f0 * e0.vx / e0.l), uy0 = g(3, v0) * -f0 + g(7, v0) * (f0 * e0.vx / e0.l);
      const double ux1 = g(2, v1) * -f1 + g(6, v1) * (f1 * e1.vx / e1.l), uy1 = g(3, v1) * -f1 + g(7, v1) * (f1 * e1.vx / e1.l);
      const double vx0 = g(4, v0) * -f0 + g(6, v0) * (f0 * e0.vy / e0.l), vy0 = g(5, v0) * -f0 + g(7, v0) * (f0 * e0.vy / e0.l);
      const double vx1 = g(4, v1) * -f1 + g(6, v1) * (f1 * e1.vy / e1.l), vy1 = g(5, v1) * -f1 + g(7, v1) * (f1 * e1.vy / e1.l);
      const double gux = ux0 * 0.5 + ux1 * 0.5, guy = uy0 * 0.5 + uy1 * 0.5;
      const double gvx = vx0 * 0.5 + vx1 * 0.5, gvy = vy0 * 0.5 + vy1 * 0.5;
      const double div = gux + gvy;
      const double sxx = 2.0 * mu * (gux - (1.0 / 3.0) * div);
      const double syy = 2.0 * mu * (gvy - (1.0 / 3.0) * div);
      const double sxy = mu * (guy + gvx);
      acc[2] += -(sxx * nx + sxy * ny);
      acc[3] += -(sxy * nx + syy * ny);
    }
  }
  __shared__ double red[4][kBlock];
#pragma unroll
  for (int c = 0; c < 4; ++c) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int o = kBlock / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
#pragma unroll
      for (int c = 0; c < 4; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int c = 0; c < 4; ++c) out[4 * f + c] = red[c][0];
}

// ------------------------------------------------------------ MC moments
// increment_moments (src/fv.cc:595-694) for the k-th sample of a group, one
// thread per vertex.  Moment arrays are [var][vertex] with the per-vertex
// record of the reference's reduce_moments packing: PrimVar (T, p, u, v, w)
// then density, mach, entropy, vorticity as selected by `extras` (bits 0-3).
// Vorticity (src/material.h:623-627) reads the entropy-variable gradients G of
// the last gradient pass: V2 = 2 beta u, V3 = 2 beta v, V5 = -2 beta.
__global__ void k_moments_increment(Params k, int nv, const double* __restrict__ P, const double* __restrict__ G,
                                    int extras, int nvar, long long kk, double* __restrict__ fm,
                                    double* __restrict__ sm, double* __restrict__ m2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  Prim q = load_prim(P, nv, i);
  double x[9];
  x[0] = q.T; x[1] = q.p; x[2] = q.u; x[3] = q.v; x[4] = 0.0;
  int j = 5;
  if (extras & 1) x[j++] = density(k, q);
  if (extras & 2) x[j++] = sqrt(q.u * q.u + q.v * q.v) / sound_speed(k, q);
  if (extras & 4) x[j++] = entropy_fn(k, q);
  if (extras & 8)
    x[j++] = k.R * q.T * (G[4 * (size_t)nv + i] + q.v * G[6 * (size_t)nv + i] - G[3 * (size_t)nv + i] -
                          q.u * G[7 * (size_t)nv + i]);
  const double K = (double)kk, c1 = 1.0 / K, c2 = (K - 1.0) / K;
  for (int c = 0; c < nvar; ++c) {
    const size_t o = (size_t)c * nv + i;
    const double xc = x[c];
    if (kk == 1) {
      fm[o] = xc; sm[o] = xc * xc; m2[o] = 0.0;
    } else {
      const double mkm1 = fm[o];
      const double mk = c < 5 ? xc * c1 + mkm1 * c2 : mkm1 + (xc - mkm1) / K;   // PrimVar::equ / scalar form
      fm[o] = mk;
      sm[o] += xc * xc;
      m2[o] += (xc - mkm1) * (xc - mk);
    }
  }
}

// One received group of reduce_moments (src/reduce_moments.cc:36-113).
__global__ void k_moments_merge(size_t n, double fact1, double fact2, double* __restrict__ fm,
                                double* __restrict__ sm, double* __restrict__ m2, const double* __restrict__ fo,
                                const double* __restrict__ so, const double* __restrict__ mo) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double diff = fo[j] - fm[j];
  fm[j] += diff * fact1;
  m2[j] += mo[j] + (diff * diff) * fact2;
  sm[j] += so[j];
}

// Final scaling of reduce_moments (src/reduce_moments.cc:115-141).
__global__ void k_moments_scale(size_t n, double fact3, double fact4, double* __restrict__ sm,
                                double* __restrict__ m2) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j >= n) return;
  m2[j] *= fact3;
  sm[j] *= fact4;
}

// ---- domain decomposition (tg_part_*): halo exchange and the exchanged step scalars

// Packs 8 doubles per listed vertex (components 0-3 of A, then 0-3 of B: the P and W
// of a state buffer, or the two halves of the gradient array) into out[8 * i + c].
__global__ void k_halo_pack(int n, const int* __restrict__ idx, int nv, const double* __restrict__ A,
                            const double* __restrict__ B, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 8 * n) return;
  const int v = idx[i >> 3], c = i & 7;
  out[i] = c < 4 ? A[(size_t)c * nv + v] : B[(size_t)(c - 4) * nv + v];
}

__global__ void k_halo_unpack(int n, const int* __restrict__ idx, int nv, double* __restrict__ A,
                              double* __restrict__ B, const double* __restrict__ in) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 8 * n) return;
  const int v = idx[i >> 3], c = i & 7;
  if (c < 4) A[(size_t)c * nv + v] = in[i];
  else B[(size_t)(c - 4) * nv + v] = in[i];
}

// After the first-stage dt pass of tg_part_prime: its minimum is the next step's.
__global__ void k_part_primed(Scalars* sc) {
  sc->dtmin_next = sc->dtmin_bits;
  sc->dtmin_bits = 0x7ff0000000000000ull;
  sc->dt_next = 1;
}

// A partition's contribution to the step exchange: its running dt minimum (as
// bits; positive doubles order like their bit patterns) and its residual-norm sums.
__global__ void k_part_export(const Scalars* sc, unsigned long long* out) {
  out[0] = sc->dtmin_next;
#pragma unroll
  for (int c = 0; c < 4; ++c) out[1 + c] = (unsigned long long)__double_as_longlong(sc->rsq[c]);
}

// All partitions' contributions, combined in partition order so every partition
// forms the same dt and norms: the dt minimum of the whole mesh and, after a
// step, the norms over the whole mesh with nv_total its vertex count (the
// reference's MPI reductions, src/fv.cc:1602, src/reduce_res_norm.cc:25).
__global__ void k_part_import(Scalars* sc, const unsigned long long* __restrict__ all, int n_parts, int nv_total,
                              int norms) {
  unsigned long long m = all[0];
  double sum4[4] = {0.0, 0.0, 0.0, 0.0};
  for (int q = 0; q < n_parts; ++q) {
    m = all[5 * q] < m ? all[5 * q] : m;
#pragma unroll
    for (int c = 0; c < 4; ++c) sum4[c] += __longlong_as_double((long long)all[5 * q + 1 + c]);
  }
  sc->dtmin_next = m;
  if (norms) set_norms(sc, sum4, nv_total, sc->iter == 1);
}

// Owned vertices of a partition -> PrimVar records in local order (tg_get_state).
__global__ void k_part_state_out(int n, int nv, const double* __restrict__ P, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double* q = out + 5 * (size_t)i;
  q[0] = P[i]; q[1] = P[3 * (size_t)nv + i]; q[2] = P[nv + i]; q[3] = P[2 * (size_t)nv + i]; q[4] = 0.0;
}

}  // namespace tg
