// tg_batch.cuh -- batched FP32 Monte Carlo ensembles: physics and kernels.
//
// An ensemble level is S samples of one mesh, advanced together.
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
//
// Meshes with walls or far field, and Navier-Stokes, add per stage a boundary
// pass (one flux per boundary-face vertex and sample) and a viscous pass (one
// set of viscous fluxes per cell or boundary face and sample), both stored and
// gathered by the vertex pass in the order of the per-vertex boundary list.
// Boundary values and the viscosity are per sample (uncertain inflow, Re).
#pragma once

#include <cstdint>

#include "tg_expr.cuh"
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
  const float* visw;               // sum over the vertex's edges of |n| / |x_b - x_a| (viscous time step)
  const double* aw;                // dual area x periodic-copy weight (integrals)
  const double *x, *y;             // coordinates (initial conditions)
  // non-periodic boundary faces and the per-vertex boundary / viscous gather
  // (entry (index << 2) | type, types as in tg_mesh.h)
  int nb, nvu, nic;                // boundary faces, viscous units, interior-cell units
  const int *b_v0, *b_v1, *b_kind, *b_adiab;
  const float *b_nx, *b_ny;
  const int *cb_off, *cb_ent;
  // viscous units: interior cells, then one boundary cell per boundary face
  const int *u_cell, *c_v;         // cell of a unit; 3 vertices per cell
  const float *c_n, *c_inv2a;      // 6 P1 normals per cell; 1 / (2 cell area)
  const int *c_bf_off, *c_bf;      // boundary faces with the cell on their left (gradient corrections)
  const int *c_nbr_off, *c_nbr;    // the cell's boundary faces in cell.face slot order
  const float *bf_nx, *bf_ny;      // face-list normal of a boundary face
  const int *bf_v0, *bf_v1;        // face-list vertex order of a boundary face
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
  // boundaries / Navier-Stokes (null on periodic Euler levels)
  float* bval;                     // nb x 10 x S: boundary values (T,u,v,w,p at face vertex 0, then 1)
  float* mu;                       // S: viscosity per sample (constant viscosity law)
  float* Fb;                       // 2 nb x 4 x S: boundary fluxes per face vertex
  float* Fv;                       // nvu x 9 x S: viscous fluxes (x, y, energy) toward the cell's 3 vertices
  float* Fvb;                      // nb x 3 x S: viscous boundary fluxes
  long long w_begin;               // first warp of this level in a fused launch (set per launch shape)
};

struct Batch {
  int nlev;
  Level lev[kMaxLevels];
  long long work;                  // warps of a fused launch over all levels
};

struct BParams {
  float gamma, R, inv_gm1, inv_gamma, sqrt_gm1, cfl, ev_alpha, ev_beta;
  float cp_over_pr;                // Cp / Pr (heat conductivity = mu Cp / Pr)
  int model, visc, heat;           // 0 Euler, 1 Navier-Stokes; viscous / heat terms active
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
                                       float& rho_ln, float& ibeta, float& p) {
  // __fdividef: at most 2 ulp for the magnitudes of densities and beta
  rho_ln = __fdividef(0.5f * (L.rho + R.rho), logavg_F_mixed(L.rho, R.rho));
  ibeta = __fdividef(logavg_F_mixed(L.beta, R.beta), 0.5f * (L.beta + R.beta));
  p = __fdividef(0.5f * (L.rho + R.rho), L.beta + R.beta);
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
// First order and minmod are positively homogeneous of degree one, so the
// eigenvector scaling S enters only squared: S (Lambda jump(S R0^T V)) =
// S^2 (Lambda jump(R0^T V)), S0^2 = rho/(2 gamma), S1^2 = (gamma-1) rho/gamma,
// S2^2 = p, without their square roots.
template <int ROE, int RECON>
__device__ __forceinline__ FFlx ftecno(const BParams& k, const FRec& L, const FRec& R, float unx, float uny, float dx,
                                       float dy, const float* gL, const float* gR) {
  static_assert(RECON == RECON_FIRST || RECON == RECON_TVD_MINMOD, "ensembles run first order or minmod");
  float rho, ibeta, p;
  FFlx F = fkepec(k, L, R, unx, uny, rho, ibeta, p);
  const float aa = 0.5f * k.gamma * ibeta;             // a^2
  const float a = sqrtf(aa);
  const float vx = 0.5f * (L.u + R.u), vy = 0.5f * (L.v + R.v);
  const float vn = vx * unx + vy * uny;
  const float vsq = vx * vx + vy * vy;
  const float H = aa * k.inv_gm1 + 0.5f * vsq;
  const float v1 = vx * uny - vy * unx;
  auto RT = [&](const float* x, float* z) {
    const float A = x[0] + vx * x[1] + vy * x[2];
    const float B = unx * x[1] + uny * x[2] + vn * x[3];
    const float C = A + H * x[3];
    z[0] = C - a * B;
    z[1] = A + (0.5f * vsq) * x[3];
    z[2] = uny * x[1] - unx * x[2] + v1 * x[3];
    z[3] = C + a * B;
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
  const float s01 = rho * k.inv_gamma;
  q[0] *= 0.5f * s01; q[1] *= (k.gamma - 1.0f) * s01; q[2] *= p; q[3] *= 0.5f * s01;
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
  float r, b, p;
  return fkepec(k, L, R, unx, uny, r, b, p);
}

// ------------------------------------------------- FP32 boundaries, viscous
struct FPrim { float T, u, v, p; };
struct FEnt { float f, vx, vy, l; };

// Primitive state of a stored record q (u, v, p, V1, V5 at stride P).
__device__ __forceinline__ FPrim fprim(const BParams& k, const float* q, int P) {
  FPrim s;
  s.u = q[0]; s.v = q[P]; s.p = q[2 * P];
  s.T = s.p / (k.R * (-q[4 * P] * s.p));
  return s;
}

__device__ __forceinline__ FEnt fprim2ent(const BParams& k, const FPrim& q) {   // src/material.h:534-546
  const float rho = q.p / (k.R * q.T);
  const float beta = rho / (2.0f * q.p);
  const float s = logf(q.p) - k.gamma * logf(rho);
  FEnt e;
  e.f = (k.gamma - s) * k.inv_gm1 - (q.u * q.u + q.v * q.v) * beta;
  e.vx = q.u * (2.0f * beta);
  e.vy = q.v * (2.0f * beta);
  e.l = -2.0f * beta;
  return e;
}

// BoundaryCondition::apply, single-state form (src/bc.h:615-654); val holds
// T, u, v, w, p of one face vertex at stride P.
__device__ __forceinline__ void fbc_apply1(int kind, int adiabatic, const float* val, int P, float nx, float ny,
                                           FPrim& s) {
  switch (kind) {
    case BC_SLIP: {
      const float im = 1.0f / sqrtf(nx * nx + ny * ny);
      const float ux = nx * im, uy = ny * im;
      const float fact = s.u * ux + s.v * uy;
      s.u += ux * -fact;
      s.v += uy * -fact;
      break;
    }
    case BC_NOSLIP:
      s.u = val[P]; s.v = val[2 * P];
      if (!adiabatic) s.T = val[0];
      break;
    case BC_PRESSURE: s.p = val[4 * P]; break;
    case BC_INLET: s.T = val[0]; s.u = val[P]; s.v = val[2 * P]; s.p = val[4 * P]; break;
    default: break;
  }
}

// Two-state form (src/bc.h:568-610): s0 the state the flux sees inside, s1 the boundary state.
__device__ __forceinline__ void fbc_apply2(int kind, int adiabatic, const float* val, int P, float nx, float ny,
                                           FPrim& s0, FPrim& s1) {
  switch (kind) {
    case BC_SLIP: {
      const float im = 1.0f / sqrtf(nx * nx + ny * ny);
      const float ux = nx * im, uy = ny * im;
      const float fact = s0.u * ux + s0.v * uy;
      s0.u += ux * -fact;
      s0.v += uy * -fact;
      s1 = s0;
      break;
    }
    case BC_NOSLIP:
      s0.u = val[P]; s0.v = val[2 * P];
      s1.u = s0.u; s1.v = s0.v;
      s1.p = s0.p;
      if (adiabatic) s1.T = s0.T;
      else { s0.T = val[0]; s1.T = val[0]; }
      break;
    case BC_PRESSURE: s1.p = val[4 * P]; break;
    case BC_INLET:
      s0.T = val[0]; s0.u = val[P]; s0.v = val[2 * P]; s0.p = val[4 * P];
      s1 = s0;
      break;
    case BC_OUTLET: s1 = s0; break;
    case BC_FARFIELD: s1.T = val[0]; s1.u = val[P]; s1.v = val[2 * P]; s1.p = val[4 * P]; break;
    default: break;
  }
}

// Entropy variables of the single-state condition applied to stored record q.
// Where the condition keeps T and p (slip, adiabatic no-slip) beta and the
// entropy are unchanged and V1 moves by beta (|u|^2 - |u'|^2) exactly; where
// it changes nothing the stored variables are returned; otherwise they are
// formed anew.
__device__ __forceinline__ FEnt fbc_ent(const BParams& k, int kind, int adiabatic, const float* val, int P, float nx,
                                        float ny, const float* q) {
  FPrim s = fprim(k, q, P);
  const float u0 = s.u, v0 = s.v;
  const float V1 = q[3 * P], V5 = q[4 * P];
  const bool keeps_Tp = kind == BC_SLIP || (kind == BC_NOSLIP && adiabatic);
  const bool changes = keeps_Tp || kind == BC_NOSLIP || kind == BC_PRESSURE || kind == BC_INLET;
  if (!changes) return FEnt{V1, -V5 * u0, -V5 * v0, V5};
  fbc_apply1(kind, adiabatic, val, P, nx, ny, s);
  if (!keeps_Tp) return fprim2ent(k, s);
  const float beta = -0.5f * V5;
  return FEnt{V1 + beta * ((u0 * u0 + v0 * v0) - (s.u * s.u + s.v * s.v)), -V5 * s.u, -V5 * s.v, V5};
}

// Flux record of a boundary state (entropy formed from T and p).
__device__ __forceinline__ FRec frec_prim(const BParams& k, const FPrim& s, bool need_a) {
  const float rho = s.p / (k.R * s.T);
  const float beta = rho / (2.0f * s.p);
  const float ent = logf(s.p) - k.gamma * logf(rho);
  const float V1 = (k.gamma - ent) * k.inv_gm1 - (s.u * s.u + s.v * s.v) * beta;
  return frec(k, s.u, s.v, s.p, V1, -2.0f * beta, need_a);
}

// Material::inviscid_bflux (src/material.cc:110-127), normal of length |n|.
__device__ __forceinline__ FFlx finviscid_bflux(const BParams& k, const FPrim& q, const FPrim& qb, float nx, float ny) {
  const float vnb = qb.u * nx + qb.v * ny;
  const float vn = q.u * nx + q.v * ny;
  const float rho = q.p / (k.R * q.T);
  FFlx F;
  F.m = rho * vnb;
  F.x = nx * qb.p + q.u * F.m;
  F.y = ny * qb.p + q.v * F.m;
  F.e = (0.5f * rho * (q.u * q.u + q.v * q.v) + k.gamma * q.p * k.inv_gm1) * vnb + (qb.p - q.p) * vn;
  return F;
}

// Viscous matrices K dV (src/material.cc:158-230) at the entropy state st for
// the cell gradient dE (V1, V2, V3, V5) x (x, y), constant viscosity mu.
struct FViscK { float a1, a2, a4, b1, b2, b4, e4, c2; };

__device__ __forceinline__ FViscK fviscous_K(const BParams& k, float mu_s, const FEnt& st, const float* dE) {
  float mu = mu_s;
  float kk = mu * k.cp_over_pr;
  if (!k.visc) mu = 0.0f;
  if (!k.heat) kk = 0.0f;
  const float e4 = 1.0f / st.l;
  const float e1 = st.vx * e4, e2 = st.vy * e4;
  const float c1 = 4.0f * mu / 3.0f, c2 = kk / k.R, c3 = 2.0f * mu / 3.0f;
  const float d1x = dE[2], d1y = dE[3], d2x = dE[4], d2y = dE[5], d4x = dE[6], d4y = dE[7];
  const float K11_1 = c1 * (-d1x + e1 * d4x);
  const float K11_2 = mu * (-d2x + e2 * d4x);
  const float K11_4 = c1 * e1 * d1x + mu * (e2 * d2x) + (-c1 * e1 * e1 - mu * (e2 * e2) + c2 * e4) * d4x;
  const float K12_1 = c3 * (d2y - e2 * d4y);
  const float K12_2 = mu * (-d1y + e1 * d4y);
  const float K12_4 = mu * e2 * d1y - c3 * e1 * d2y - (mu - c3) * e1 * e2 * d4y;
  const float K21_1 = mu * (-d2x + e2 * d4x);
  const float K21_2 = c3 * (d1x - e1 * d4x);
  const float K21_4 = -c3 * e2 * d1x + mu * e1 * d2x - (mu - c3) * e1 * e2 * d4x;
  const float K22_1 = mu * (-d1y + e1 * d4y);
  const float K22_2 = c1 * (-d2y + e2 * d4y);
  const float K22_4 = mu * (e1 * d1y) + c1 * e2 * d2y + (-mu * (e1 * e1) - c1 * e2 * e2 + c2 * e4) * d4y;
  FViscK r;
  r.a1 = K11_1 + K12_1; r.a2 = K11_2 + K12_2; r.a4 = K11_4 + K12_4;
  r.b1 = K21_1 + K22_1; r.b2 = K21_2 + K22_2; r.b4 = K21_4 + K22_4;
  r.e4 = e4;
  r.c2 = c2;
  return r;
}

__device__ __forceinline__ void fviscous_apply(const FViscK& K, float nx, float ny, float& fx, float& fy, float& fe) {
  fx = -(K.a1 * nx + K.b1 * ny) * K.e4;
  fy = -(K.a2 * nx + K.b2 * ny) * K.e4;
  fe = -(K.a4 * nx + K.b4 * ny) * K.e4;
}

// ------------------------------------------------------------ paired samples
// The three per-stage kernels over vertices and edges (gradients, edge fluxes,
// gather + RK stage) hold two neighbouring samples per thread: one 8-byte load
// per stored pair, the index and address work shared by the pair, and the FP32
// arithmetic issued as paired instructions (__fadd2_rn, __fmul2_rn, __ffma2_rn:
// each component rounds as the scalar _rn operation does).  What has no paired
// form runs per component: reciprocals and square roots of the flux (the
// approximate forms, at most 1 ulp and 2^-23 relative, as __fdividef), the
// logarithms, the FP64 near-equal branch of the log mean and the limiter's
// selects.  A sample's arithmetic is the same whichever sample it is paired
// with and whatever the launch shape.
typedef float2 f2;
__device__ __forceinline__ f2 sp(float a) { return make_float2(a, a); }
__device__ __forceinline__ f2 neg2(f2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ f2 add2(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 sub2(f2 a, f2 b) { return __fadd2_rn(a, neg2(b)); }
__device__ __forceinline__ f2 mul2(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ f2 abs2(f2 a) { return make_float2(fabsf(a.x), fabsf(a.y)); }
__device__ __forceinline__ float rcp_apx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float sqrt_apx(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ f2 rcp2(f2 a) { return make_float2(rcp_apx(a.x), rcp_apx(a.y)); }
__device__ __forceinline__ f2 sqrt2(f2 a) { return make_float2(sqrt_apx(a.x), sqrt_apx(a.y)); }
__device__ __forceinline__ f2 ld2(const float* p) { return __ldg(reinterpret_cast<const float2*>(p)); }
__device__ __forceinline__ void st2(float* p, f2 v) { *reinterpret_cast<float2*>(p) = v; }

// F of the Ismail-Roe log mean of one component (src/material.h:24-42), the
// near-equal series in FP64; 1 / (a + b) from the approximate FP32 reciprocal
// refined by one Newton-Raphson step in FP64 (relative error about 2^-46).
__device__ __forceinline__ float logF1(float a, float b) {
  const double da = a, db = b;
  const double d = db + da;                      // exact in FP64, as is db - da
  const double y0 = (double)rcp_apx((float)d);
  const double f = (db - da) * (y0 * ::fma(-d, y0, 2.0));
  const double u = f * f;
  if (u < 1.0e-2) {
    const double u2 = u * u;
    return (float)::fma(u2 * u, 1.0 / 7.0, ::fma(u2, 1.0 / 5.0, ::fma(u, 1.0 / 3.0, 1.0)));
  }
  return logf(b / a) / (2.0f * (float)f);
}

// minmod (src/limiter.h:14-27) of one component
__device__ __forceinline__ float minmod1(float a, float b) {
  const float m = fminf(fabsf(a), fabsf(b));
  return ((a > 0.0f && b > 0.0f) || (a < 0.0f && b < 0.0f)) ? copysignf(m, a) : 0.0f;
}

struct PRec { f2 rho, u, v, p, beta, V1; };
struct PFlx { f2 m, x, y, e; };
struct PAvg { f2 rho, ibeta, p, vx, vy, vn; };

// Flux record from a stored pair (u, v, p, V1, V5 with V5 = -2 beta, rho = 2 beta p).
__device__ __forceinline__ PRec prec(f2 u, f2 v, f2 p, f2 V1, f2 V5) {
  PRec r;
  const f2 nV5 = neg2(V5);
  r.u = u; r.v = v; r.p = p; r.V1 = V1;
  r.beta = mul2(sp(0.5f), nV5);
  r.rho = mul2(nV5, p);
  return r;
}

// KEPEC central flux (src/kepec.cc:10-38) on a unit normal, with its averages.
__device__ __forceinline__ PFlx kepec2(const BParams& k, const PRec& L, const PRec& R, float unx, float uny, PAvg& A) {
  const f2 sr = add2(L.rho, R.rho), sb = add2(L.beta, R.beta);
  const f2 Fr = make_float2(logF1(L.rho.x, R.rho.x), logF1(L.rho.y, R.rho.y));
  const f2 Fb = make_float2(logF1(L.beta.x, R.beta.x), logF1(L.beta.y, R.beta.y));
  const f2 hs = mul2(sp(0.5f), sr);
  const f2 isb = rcp2(sb);
  A.rho = mul2(hs, rcp2(Fr));          // (rho_l + rho_r) / 2 / F_rho
  A.p = mul2(hs, isb);                 // (rho_l + rho_r) / (2 (beta_l + beta_r))
  A.ibeta = mul2(add2(Fb, Fb), isb);   // F_beta / ((beta_l + beta_r) / 2)
  A.vx = mul2(sp(0.5f), add2(L.u, R.u));
  A.vy = mul2(sp(0.5f), add2(L.v, R.v));
  A.vn = fma2(A.vy, sp(uny), mul2(A.vx, sp(unx)));
  const f2 vel2 = mul2(sp(0.5f), add2(fma2(L.v, L.v, mul2(L.u, L.u)), fma2(R.v, R.v, mul2(R.u, R.u))));
  PFlx F;
  F.m = mul2(A.rho, A.vn);
  F.x = fma2(A.vx, F.m, mul2(sp(unx), A.p));
  F.y = fma2(A.vy, F.m, mul2(sp(uny), A.p));
  const f2 h = mul2(sp(0.5f), fma2(A.ibeta, sp(k.inv_gm1), neg2(vel2)));
  F.e = fma2(h, F.m, fma2(F.y, A.vy, mul2(F.x, A.vx)));
  return F;
}

// KEPES-TeCNO (src/kepes_tecno_roe.cc:11-173, src/kepes_tecno_rusanov.cc:11-164)
// in the unscaled form of ftecno: S^2 (Lambda jump(R0^T V)), first order or minmod.
template <int ROE, int RECON>
__device__ __forceinline__ PFlx tecno2(const BParams& k, const PRec& L, const PRec& R, float unx, float uny, float dx,
                                       float dy, const f2* gL, const f2* gR) {
  static_assert(RECON == RECON_FIRST || RECON == RECON_TVD_MINMOD, "ensembles run first order or minmod");
  PAvg A;
  PFlx F = kepec2(k, L, R, unx, uny, A);
  const f2 U = sp(unx), W = sp(uny);
  const f2 aa = mul2(sp(0.5f * k.gamma), A.ibeta);   // a^2
  const f2 a = sqrt2(aa);
  const f2 hv = mul2(sp(0.5f), fma2(A.vy, A.vy, mul2(A.vx, A.vx)));
  const f2 H = fma2(aa, sp(k.inv_gm1), hv);
  const f2 v1 = fma2(A.vx, W, mul2(A.vy, sp(-unx)));
  auto RT = [&](const f2* x, f2* z) {
    const f2 Aq = fma2(A.vy, x[2], fma2(A.vx, x[1], x[0]));
    const f2 Bq = fma2(A.vn, x[3], fma2(W, x[2], mul2(U, x[1])));
    const f2 Cq = fma2(H, x[3], Aq);
    z[0] = fma2(neg2(a), Bq, Cq);
    z[1] = fma2(hv, x[3], Aq);
    z[2] = fma2(v1, x[3], fma2(W, x[1], mul2(sp(-unx), x[2])));
    z[3] = fma2(a, Bq, Cq);
  };
  f2 Lam[4];
  if (ROE) {
    const f2 gr = sp(k.gamma);
    const f2 al = sqrt2(mul2(mul2(gr, L.p), rcp2(L.rho))), ar = sqrt2(mul2(mul2(gr, R.p), rcp2(R.rho)));
    const f2 vnl = fma2(L.v, W, mul2(L.u, U)), vnr = fma2(R.v, W, mul2(R.u, U));
    const f2 b1 = sp(1.0f + k.ev_beta), al1 = sp(k.ev_alpha);
    Lam[0] = fma2(b1, abs2(sub2(A.vn, a)), mul2(al1, abs2(sub2(sub2(vnl, al), sub2(vnr, ar)))));
    Lam[1] = Lam[2] = abs2(A.vn);
    Lam[3] = fma2(b1, abs2(add2(A.vn, a)), mul2(al1, abs2(sub2(add2(vnl, al), add2(vnr, ar)))));
  } else {
    Lam[0] = Lam[1] = Lam[2] = Lam[3] = add2(abs2(A.vn), a);
  }
  // V = (V1, 2 beta u, 2 beta v, -2 beta)
  f2 dV[4];
  dV[0] = sub2(R.V1, L.V1);
  dV[1] = mul2(sp(2.0f), fma2(R.u, R.beta, neg2(mul2(L.u, L.beta))));
  dV[2] = mul2(sp(2.0f), fma2(R.v, R.beta, neg2(mul2(L.v, L.beta))));
  dV[3] = mul2(sp(-2.0f), sub2(R.beta, L.beta));
  f2 q[4];
  RT(dV, q);
  if (RECON != RECON_FIRST) {
    f2 gl[4], gr[4], sl[4], sr[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      gl[i] = fma2(gL[2 * i + 1], sp(dy), mul2(gL[2 * i], sp(dx)));
      gr[i] = fma2(gR[2 * i + 1], sp(dy), mul2(gR[2 * i], sp(dx)));
    }
    RT(gl, sl);
    RT(gr, sr);
#pragma unroll
    for (int i = 0; i < 4; ++i) {   // Z_ji - Z_ij = d - minmod(2 s_r - d, d) / 2 - minmod(2 s_l - d, d) / 2
      const f2 d = q[i], nd = neg2(d);
      const f2 xr = fma2(sp(2.0f), sr[i], nd), xl = fma2(sp(2.0f), sl[i], nd);
      const f2 mr = make_float2(minmod1(xr.x, d.x), minmod1(xr.y, d.y));
      const f2 ml = make_float2(minmod1(xl.x, d.x), minmod1(xl.y, d.y));
      q[i] = fma2(sp(-0.5f), ml, fma2(sp(-0.5f), mr, d));
    }
  }
  const f2 s01 = mul2(A.rho, sp(k.inv_gamma));
  const f2 hs01 = mul2(sp(0.5f), s01);
  q[0] = mul2(mul2(Lam[0], q[0]), hs01);
  q[1] = mul2(mul2(Lam[1], q[1]), mul2(sp(k.gamma - 1.0f), s01));
  q[2] = mul2(mul2(Lam[2], q[2]), A.p);
  q[3] = mul2(mul2(Lam[3], q[3]), hs01);
  const f2 sum = add2(add2(q[0], q[1]), q[3]), dif = sub2(q[3], q[0]);
  const f2 adif = mul2(a, dif), mh = sp(-0.5f);
  F.m = fma2(mh, sum, F.m);
  F.x = fma2(mh, fma2(W, q[2], fma2(adif, U, mul2(A.vx, sum))), F.x);
  F.y = fma2(mh, fma2(sp(-unx), q[2], fma2(adif, W, mul2(A.vy, sum))), F.y);
  F.e = fma2(mh, fma2(v1, q[2], fma2(hv, q[1], fma2(adif, A.vn, mul2(H, add2(q[0], q[3]))))), F.e);
  return F;
}

template <int FLUX, int RECON>
__device__ __forceinline__ PFlx pflux(const BParams& k, const PRec& L, const PRec& R, float unx, float uny, float dx,
                                      float dy, const f2* gL, const f2* gR) {
  if (FLUX == FLUX_TECNO_ROE) return tecno2<1, RECON>(k, L, R, unx, uny, dx, dy, gL, gR);
  if (FLUX == FLUX_TECNO_RUSANOV) return tecno2<0, RECON>(k, L, R, unx, uny, dx, dy, gL, gR);
  PAvg A;
  return kepec2(k, L, R, unx, uny, A);
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

// What a launch's items are: (vertex | edge | boundary-face vertex | viscous unit, sample).
enum : int { IT_VERTEX = 0, IT_EDGE = 1, IT_BSLOT = 2, IT_UNIT = 3 };

__host__ __device__ __forceinline__ int item_count(const LevelMesh& m, int kind) {
  return kind == IT_VERTEX ? m.nv : kind == IT_EDGE ? m.ne : kind == IT_BSLOT ? 2 * m.nb : m.nvu;
}

// The warp index of a launch fits 32 bits (tg_batch_create refuses larger
// batches), so the split into sample tile and item warp is a 32-bit division.
template <int ST, int KIND = IT_VERTEX>
__device__ __forceinline__ Item item_of(const Batch& B, unsigned w, int lane) {
  constexpr unsigned VPW = 32 / ST;
  Item it{0, 0, 0, false};
  if ((long long)w >= B.work) return it;
  int l = 0;
#pragma unroll
  for (int i = 1; i < kMaxLevels; ++i)
    if (i < B.nlev && (long long)w >= B.lev[i].w_begin) l = i;
  const unsigned r = w - (unsigned)B.lev[l].w_begin;
  const unsigned n = (unsigned)item_count(B.lev[l].m, KIND);
  const unsigned nvw = (n + VPW - 1) / VPW;
  const unsigned tile = r / nvw;
  it.l = l;
  it.s = (int)(tile * ST) + (lane % ST);
  it.v = (int)((r - tile * nvw) * VPW) + lane / ST;
  it.ok = it.v < (int)n;
  return it;
}

// Paired kernels (gradients, edge fluxes, gather + update): each lane holds H
// pairs of neighbouring samples, ST / (2 H) lanes per item, so a warp covers
// 64 H / ST items x ST samples.
template <int ST, int H = 1>
__host__ __device__ __forceinline__ long long level_warps_pair(int nv, int S) {
  constexpr int IPW = 64 * H / ST;
  return (long long)((nv + IPW - 1) / IPW) * (S / ST);
}

template <int ST, int KIND = IT_VERTEX, int H = 1>
__device__ __forceinline__ Item item_of_pair(const Batch& B, unsigned w, int lane) {
  constexpr unsigned LPI = ST / (2 * H), IPW = 64 * H / ST;
  static_assert(LPI >= 1, "sample tile too small for the pairs per lane");
  Item it{0, 0, 0, false};
  if ((long long)w >= B.work) return it;
  int l = 0;
#pragma unroll
  for (int i = 1; i < kMaxLevels; ++i)
    if (i < B.nlev && (long long)w >= B.lev[i].w_begin) l = i;
  const unsigned r = w - (unsigned)B.lev[l].w_begin;
  const unsigned n = (unsigned)item_count(B.lev[l].m, KIND);
  const unsigned nvw = (n + IPW - 1) / IPW;
  const unsigned tile = r / nvw;
  it.l = l;
  it.s = (int)(tile * ST) + 2 * H * (int)(lane % LPI);
  it.v = (int)((r - tile * nvw) * IPW) + (int)(lane / LPI);
  it.ok = it.v < (int)n;
  return it;
}

// Pairs per lane of the gradient and gather passes.
#ifndef TG_BATCH_LANE_PAIRS
#define TG_BATCH_LANE_PAIRS 2
#endif
constexpr int kLanePairs = TG_BATCH_LANE_PAIRS;

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

// Local time step (src/fv.cc:1499-1580) of every vertex and the running
// per-sample minimum; U_old (src/fv.cc:1626-1630).  Each lane keeps a pair of
// samples (a group of 64; the last group of a level whose sample count is an
// odd multiple of 32 leaves its upper half-warp idle) and walks a strided set of
// vertices, so one atomic per block and sample remains.  BND adds the
// boundary-face terms and, for Navier-Stokes, the viscous ones, in the
// reference's order.
__host__ __device__ __forceinline__ int dt_groups(int S) { return (S + 63) / 64; }

template <int VT, bool BND>
__global__ void __launch_bounds__(32 * VT) kb_dt(Batch B, BParams k, int chunks) {
  const int lane = threadIdx.x & 31, vg = threadIdx.x >> 5;
  // blockIdx.x: (level, sample group, chunk)
  long long bid = blockIdx.x;
  int l = 0;
  long long base = 0;
  for (int i = 0; i < B.nlev; ++i) {
    const long long nb = (long long)dt_groups(B.lev[i].S) * chunks;
    if (bid < base + nb) { l = i; break; }
    base += nb;
  }
  const Level& L = B.lev[l];
  const int r = (int)(bid - base);
  const int sg = r / chunks, ch = r - sg * chunks;
  const int s = sg * 64 + 2 * lane;
  const int2 act = s < L.S ? *reinterpret_cast<const int2*>(L.c.active + s) : make_int2(0, 0);
  const float inf = __int_as_float(0x7f800000);
  f2 m = sp(inf);
  if (act.x || act.y) {
    const int P = L.P;
    const int per = (L.m.nv + chunks - 1) / chunks;
    const int v0 = ch * per, v1 = min(L.m.nv, v0 + per);
    const f2 mu = BND && k.model == 1 ? make_float2(L.mu[s], L.mu[s + 1]) : sp(0.0f);
    for (int v = v0 + vg; v < v1; v += VT) {
      const float* q = L.Q[0] + rows(v, kQ, P) + s;
      const f2 u = ld2(q), w = ld2(q + P), p = ld2(q + 2 * P), V5 = ld2(q + 4 * P);
      const f2 rho = mul2(neg2(V5), p);
      const f2 gp = mul2(sp(k.gamma), p);
      const f2 c = make_float2(sqrtf(gp.x / rho.x), sqrtf(gp.y / rho.y));
      f2 lam = sp(0.0f);
      for (int j = L.m.ce_off[v]; j < L.m.ce_off[v + 1]; ++j) {
        const int e = L.m.ce_ent[j] >> 1;
        const f2 vn = fma2(w, sp(L.m.ny[e]), mul2(u, sp(L.m.nx[e])));
        lam = add2(lam, fma2(c, sp(L.m.ar[e]), abs2(vn)));
      }
      if (BND) {
        for (int j = L.m.cb_off[v]; j < L.m.cb_off[v + 1]; ++j) {
          const int ent = L.m.cb_ent[j];
          if ((ent & 3) != 0) continue;
          const int d = ent >> 3;           // entry (2 d + vertex slot) << 2
          const float nx = L.m.b_nx[d], ny = L.m.b_ny[d];
          const f2 vn = fma2(w, sp(ny), mul2(u, sp(nx)));
          lam = fma2(sp(0.5f), fma2(c, sp(sqrtf(nx * nx + ny * ny)), abs2(vn)), lam);
        }
        // the viscous terms mu |n_e| / |d_e| / rho summed over the vertex's edges, the
        // geometric sum formed once per mesh
        if (k.model == 1) lam = fma2(make_float2(mu.x / rho.x, mu.y / rho.y), sp(L.m.visw[v]), lam);
      }
      const float ca = k.cfl * L.m.area[v];
      const f2 dtv = make_float2(ca / lam.x, ca / lam.y);
      m.x = fminf(m.x, dtv.x > 0.0f ? dtv.x : inf);
      m.y = fminf(m.y, dtv.y > 0.0f ? dtv.y : inf);
      // U_old
      float* uo = L.Uold + rows(v, 4, P) + s;
      st2(uo, rho);
      st2(uo + P, mul2(rho, u));
      st2(uo + 2 * P, mul2(rho, w));
      st2(uo + 3 * P, fma2(p, sp(k.inv_gm1), mul2(mul2(sp(0.5f), fma2(w, w, mul2(u, u))), rho)));
    }
  }
  __shared__ float2 red[VT][32];
  red[vg][lane] = m;
  __syncthreads();
  if (vg == 0) {
    for (int i = 1; i < VT; ++i) {
      m.x = fminf(m.x, red[i][lane].x);
      m.y = fminf(m.y, red[i][lane].y);
    }
    if (act.x) atomicMin(&L.c.dtmin_bits[s], __float_as_uint(m.x));
    if (act.y) atomicMin(&L.c.dtmin_bits[s + 1], __float_as_uint(m.y));
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
// grad_v = sum_e g_{v,e} (W_o - W_v) / (6 mcarea)), one vertex and H pairs of
// samples per thread.  BND adds the boundary-face corrections
// n_b (W_b0 + W_b1 - W_0 - W_1) / 2 (src/fv.cc:926-966).  every != 0: all
// samples, held ones included (forces); otherwise a thread whose samples are
// all held skips.
template <int ST, bool BND, int H = BND ? 1 : kLanePairs>
__global__ void kb_grad(Batch B, BParams k, int r, int every) {
  const unsigned w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const Item it = item_of_pair<ST, IT_VERTEX, H>(B, w, threadIdx.x & 31);
  if (!it.ok) return;
  const Level& L = B.lev[it.l];
  const int v = it.v, s = it.s;
  if (!every) {
    bool any = false;
#pragma unroll
    for (int h = 0; h < H; ++h) {
      const int2 act = *reinterpret_cast<const int2*>(L.c.active + s + 2 * h);
      any = any || act.x || act.y;
    }
    if (!any) return;
  }
  const int S = L.P;   // row pitch
  const float* Q = L.Q[r] + s;
  auto W = [&](int x, f2 (*o)[4]) {   // V2 = 2 beta u = -V5 u
    const float* q = Q + rows(x, kQ, S);
#pragma unroll
    for (int h = 0; h < H; ++h) {
      const f2 V5 = ld2(q + 4 * S + 2 * h), nV5 = neg2(V5);
      o[h][0] = ld2(q + 3 * S + 2 * h); o[h][1] = mul2(nV5, ld2(q + 2 * h)); o[h][2] = mul2(nV5, ld2(q + S + 2 * h));
      o[h][3] = V5;
    }
  };
  f2 ws[H][4];
  W(v, ws);
  f2 acc[H][kG];
#pragma unroll
  for (int h = 0; h < H; ++h)
#pragma unroll
    for (int c = 0; c < kG; ++c) acc[h][c] = sp(0.0f);
  for (int j = L.m.ce_off[v]; j < L.m.ce_off[v + 1]; ++j) {
    const int ent = L.m.ce_ent[j], e = ent >> 1, side = ent & 1;
    const int o = side ? L.m.e_a[e] : L.m.e_b[e];
    const f2 gx = sp(side ? L.m.g1x[e] : L.m.g0x[e]), gy = sp(side ? L.m.g1y[e] : L.m.g0y[e]);
    f2 wo[H][4];
    W(o, wo);
#pragma unroll
    for (int h = 0; h < H; ++h)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const f2 d = sub2(wo[h][c], ws[h][c]);
        acc[h][2 * c] = fma2(gx, d, acc[h][2 * c]);
        acc[h][2 * c + 1] = fma2(gy, d, acc[h][2 * c + 1]);
      }
  }
  if (BND) {
    for (int j = L.m.cb_off[v]; j < L.m.cb_off[v + 1]; ++j) {
      const int ent = L.m.cb_ent[j];
      if ((ent & 3) != 1) continue;
      const int d = ent >> 2;
      const int kind = L.m.b_kind[d], ad = L.m.b_adiab[d];
      const float nx = L.m.b_nx[d], ny = L.m.b_ny[d];
      const float* val = L.bval + rows(d, 10, S) + s;
      const float* q0 = Q + rows(L.m.b_v0[d], kQ, S);
      const float* q1 = Q + rows(L.m.b_v1[d], kQ, S);
      f2 w0[H][4], w1[H][4];
      W(L.m.b_v0[d], w0);
      W(L.m.b_v1[d], w1);
#pragma unroll
      for (int h = 0; h < H; ++h) {
        FEnt e0[2], e1[2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const int o = 2 * h + c;
          e0[c] = fbc_ent(k, kind, ad, val + o, S, nx, ny, q0 + o);
          e1[c] = fbc_ent(k, kind, ad, val + 5 * S + o, S, nx, ny, q1 + o);
        }
        const f2 eb[4] = {add2(make_float2(e0[0].f, e0[1].f), make_float2(e1[0].f, e1[1].f)),
                          add2(make_float2(e0[0].vx, e0[1].vx), make_float2(e1[0].vx, e1[1].vx)),
                          add2(make_float2(e0[0].vy, e0[1].vy), make_float2(e1[0].vy, e1[1].vy)),
                          add2(make_float2(e0[0].l, e0[1].l), make_float2(e1[0].l, e1[1].l))};
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const f2 dW = mul2(sub2(sub2(eb[c], w0[h][c]), w1[h][c]), sp(0.5f));
          acc[h][2 * c] = fma2(sp(nx), dW, acc[h][2 * c]);
          acc[h][2 * c + 1] = fma2(sp(ny), dW, acc[h][2 * c + 1]);
        }
      }
    }
  }
  const f2 f = sp(L.m.inv6mc[v]);
  float* G = L.G + rows(v, kG, S) + s;
#pragma unroll
  for (int h = 0; h < H; ++h)
#pragma unroll
    for (int c = 0; c < kG; ++c) st2(G + c * S + 2 * h, mul2(acc[h][c], f));
}

// Edge fluxes of one stage (src/fv.cc:1066-1192, src/material.cc:27-74): one
// edge and a pair of samples per thread, the flux of the edge's own
// orientation (a left, b right) times |n|, stored for the gather.  A pair
// whose two samples are both held skips.
// Resident threads per SM the edge pass is compiled for (0: the compiler's choice).
#ifndef TG_BATCH_EDGE_THREADS
#define TG_BATCH_EDGE_THREADS 896
#endif
#if TG_BATCH_EDGE_THREADS > 0
#define TG_EDGE_BOUNDS(BS) __launch_bounds__(BS, TG_BATCH_EDGE_THREADS / (BS))
#else
#define TG_EDGE_BOUNDS(BS) __launch_bounds__(BS)
#endif
template <int FLUX, int RECON, int ST, int BS>
__global__ void TG_EDGE_BOUNDS(BS) kb_edge_flux(Batch B, BParams k, int r) {
  const unsigned w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const Item it = item_of_pair<ST, IT_EDGE>(B, w, threadIdx.x & 31);
  if (!it.ok) return;
  const Level& L = B.lev[it.l];
  const int e = it.v, s = it.s;
  const int2 act = *reinterpret_cast<const int2*>(L.c.active + s);
  if (!act.x && !act.y) return;
  constexpr bool kGr = (RECON != RECON_FIRST) && (FLUX == FLUX_TECNO_ROE || FLUX == FLUX_TECNO_RUSANOV);
  const int S = L.P;   // row pitch
  const int ia = L.m.e_a[e], ib = L.m.e_b[e];
  const float* qa = L.Q[r] + rows(ia, kQ, S) + s;
  const float* qb = L.Q[r] + rows(ib, kQ, S) + s;
  const PRec A = prec(ld2(qa), ld2(qa + S), ld2(qa + 2 * S), ld2(qa + 3 * S), ld2(qa + 4 * S));
  const PRec Bv = prec(ld2(qb), ld2(qb + S), ld2(qb + 2 * S), ld2(qb + 3 * S), ld2(qb + 4 * S));
  f2 ga[kG], gb[kG];
  if (kGr) {
    const float* Ga = L.G + rows(ia, kG, S) + s;
    const float* Gb = L.G + rows(ib, kG, S) + s;
#pragma unroll
    for (int c = 0; c < kG; ++c) { ga[c] = ld2(Ga + c * S); gb[c] = ld2(Gb + c * S); }
  } else {
#pragma unroll
    for (int c = 0; c < kG; ++c) ga[c] = gb[c] = sp(0.0f);
  }
  const PFlx F = pflux<FLUX, RECON>(k, A, Bv, L.m.ux[e], L.m.uy[e], L.m.dx[e], L.m.dy[e], ga, gb);
  const f2 ar = sp(L.m.ar[e]);
  float* Fo = L.F + rows(e, 4, S) + s;
  st2(Fo, mul2(F.m, ar)); st2(Fo + S, mul2(F.x, ar)); st2(Fo + 2 * S, mul2(F.y, ar)); st2(Fo + 3 * S, mul2(F.e, ar));
}

// Boundary-face fluxes (src/fv.cc:1100-1188): one (face vertex, sample) per
// thread.  Far field: the interior flux against the boundary state, first
// order (the reference passes zero gradients); otherwise inviscid_bflux.
template <int FLUX, int ST, int BS>
__global__ void __launch_bounds__(BS) kb_bflux(Batch B, BParams k, int r) {
  const unsigned w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const Item it = item_of<ST, IT_BSLOT>(B, w, threadIdx.x & 31);
  if (!it.ok) return;
  const Level& L = B.lev[it.l];
  const int t = it.v, s = it.s;
  if (!L.c.active[s]) return;
  constexpr bool kA = (FLUX == FLUX_TECNO_ROE);
  const int S = L.P;   // row pitch
  const int d = t >> 1, q = t & 1;
  const int c = q ? L.m.b_v1[d] : L.m.b_v0[d];
  const float* Q = L.Q[r] + rows(c, kQ, S) + s;
  FPrim s0 = fprim(k, Q, S), s1 = s0;
  const float nx = L.m.b_nx[d], ny = L.m.b_ny[d];
  const int kind = L.m.b_kind[d];
  fbc_apply2(kind, L.m.b_adiab[d], L.bval + rows(d, 10, S) + 5 * q * S + s, S, nx, ny, s0, s1);
  FFlx F;
  if (kind == BC_FARFIELD) {
    // the far-field condition leaves the interior state as stored
    const float ar = sqrtf(nx * nx + ny * ny), ia = 1.0f / ar;
    const FRec A = frec(k, Q[0], Q[S], Q[2 * S], Q[3 * S], Q[4 * S], kA);
    const FRec G = frec_prim(k, s1, kA);
    float z[kG];
#pragma unroll
    for (int i = 0; i < kG; ++i) z[i] = 0.0f;
    F = fflux<FLUX, RECON_FIRST>(k, A, G, nx * ia, ny * ia, 0.0f, 0.0f, z, z);
    F.m *= ar; F.x *= ar; F.y *= ar; F.e *= ar;
  } else {
    F = finviscid_bflux(k, s0, s1, nx, ny);
  }
  float* Fo = L.Fb + rows(t, 4, S) + s;
  Fo[0] = F.m; Fo[S] = F.x; Fo[2 * S] = F.y; Fo[3 * S] = F.e;
}

// Viscous units (src/fv.cc:1197-1320): per cell, the P1 gradient of the
// entropy variables with boundary corrections in face order, the mean entropy
// state (interior cells: the three vertices; boundary cells: the boundary
// states of the cell's boundary-face vertices), and the viscous flux through
// each vertex's P1 normal; a boundary unit adds the face's viscous flux with
// the adiabatic heat-flux correction.  One unit and a pair of samples per
// thread; boundary states per component (fbc_ent), the rest paired.
struct PViscK { f2 a1, a2, a4, b1, b2, b4, e4, c2; };

// Viscous matrices K dV (src/material.cc:158-230) for a pair, as fviscous_K.
__device__ __forceinline__ PViscK pviscous_K(const BParams& k, f2 mu, f2 vx, f2 vy, f2 l, const f2* dE) {
  f2 kk = mul2(mu, sp(k.cp_over_pr));
  if (!k.visc) mu = sp(0.0f);
  if (!k.heat) kk = sp(0.0f);
  const f2 e4 = make_float2(1.0f / l.x, 1.0f / l.y);
  const f2 e1 = mul2(vx, e4), e2 = mul2(vy, e4);
  const f2 c1 = make_float2(4.0f * mu.x / 3.0f, 4.0f * mu.y / 3.0f);
  const f2 c2 = make_float2(kk.x / k.R, kk.y / k.R);
  const f2 c3 = make_float2(2.0f * mu.x / 3.0f, 2.0f * mu.y / 3.0f);
  const f2 d1x = dE[2], d1y = dE[3], d2x = dE[4], d2y = dE[5], d4x = dE[6], d4y = dE[7];
  const f2 c1e1 = mul2(c1, e1), c1e2 = mul2(c1, e2), mue1 = mul2(mu, e1), mue2 = mul2(mu, e2);
  const f2 mmc = mul2(mul2(sub2(mu, c3), e1), e2);            // (mu - c3) e1 e2
  const f2 c2e4 = mul2(c2, e4);
  const f2 K11_1 = mul2(c1, fma2(e1, d4x, neg2(d1x)));
  const f2 K11_2 = mul2(mu, fma2(e2, d4x, neg2(d2x)));
  const f2 K11_4 = fma2(add2(sub2(neg2(mul2(c1e1, e1)), mul2(mu, mul2(e2, e2))), c2e4), d4x,
                        add2(mul2(c1e1, d1x), mul2(mu, mul2(e2, d2x))));
  const f2 K12_1 = mul2(c3, fma2(neg2(e2), d4y, d2y));
  const f2 K12_2 = mul2(mu, fma2(e1, d4y, neg2(d1y)));
  const f2 K12_4 = sub2(sub2(mul2(mue2, d1y), mul2(mul2(c3, e1), d2y)), mul2(mmc, d4y));
  const f2 K21_2 = mul2(c3, fma2(neg2(e1), d4x, d1x));
  const f2 K21_4 = sub2(add2(neg2(mul2(mul2(c3, e2), d1x)), mul2(mue1, d2x)), mul2(mmc, d4x));
  const f2 K22_2 = mul2(c1, fma2(e2, d4y, neg2(d2y)));
  const f2 K22_4 = fma2(add2(sub2(neg2(mul2(mu, mul2(e1, e1))), mul2(c1e2, e2)), c2e4), d4y,
                        add2(mul2(mu, mul2(e1, d1y)), mul2(c1e2, d2y)));
  PViscK r;
  r.a1 = add2(K11_1, K12_1); r.a2 = add2(K11_2, K12_2); r.a4 = add2(K11_4, K12_4);
  r.b1 = add2(K11_2, K12_2);                                  // K21_1 = K11_2, K22_1 = K12_2
  r.b2 = add2(K21_2, K22_2); r.b4 = add2(K21_4, K22_4);
  r.e4 = e4;
  r.c2 = c2;
  return r;
}

__device__ __forceinline__ void pviscous_apply(const PViscK& K, float nx, float ny, f2& fx, f2& fy, f2& fe) {
  const f2 me4 = neg2(K.e4), X = sp(nx), Y = sp(ny);
  fx = mul2(fma2(K.b1, Y, mul2(K.a1, X)), me4);
  fy = mul2(fma2(K.b2, Y, mul2(K.a2, X)), me4);
  fe = mul2(fma2(K.b4, Y, mul2(K.a4, X)), me4);
}

template <int ST, int BS>
__global__ void __launch_bounds__(BS) kb_viscous(Batch B, BParams k, int r) {
  const unsigned w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const Item it = item_of_pair<ST, IT_UNIT>(B, w, threadIdx.x & 31);
  if (!it.ok) return;
  const Level& L = B.lev[it.l];
  const int u = it.v, s = it.s;
  const int2 act = *reinterpret_cast<const int2*>(L.c.active + s);
  if (!act.x && !act.y) return;
  const int S = L.P;   // row pitch
  const float* Q = L.Q[r] + s;
  auto W = [&](int x, f2* o) {   // V2 = 2 beta u = -V5 u
    const float* q = Q + rows(x, kQ, S);
    const f2 V5 = ld2(q + 4 * S), nV5 = neg2(V5);
    o[0] = ld2(q + 3 * S); o[1] = mul2(nV5, ld2(q)); o[2] = mul2(nV5, ld2(q + S)); o[3] = V5;
  };
  const int c = L.m.u_cell[u];
  const float* n = L.m.c_n + 6 * (size_t)c;
  f2 wv[3][4];
#pragma unroll
  for (int i = 0; i < 3; ++i) W(L.m.c_v[3 * c + i], wv[i]);
  f2 dE[kG];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    dE[2 * i] = fma2(sp(n[4]), wv[2][i], fma2(sp(n[2]), wv[1][i], mul2(sp(n[0]), wv[0][i])));
    dE[2 * i + 1] = fma2(sp(n[5]), wv[2][i], fma2(sp(n[3]), wv[1][i], mul2(sp(n[1]), wv[0][i])));
  }
  for (int j = L.m.c_bf_off[c]; j < L.m.c_bf_off[c + 1]; ++j) {
    const int d = L.m.c_bf[j];
    const int kind = L.m.b_kind[d], ad = L.m.b_adiab[d];
    const float nx = L.m.b_nx[d], ny = L.m.b_ny[d];
    const float* val = L.bval + rows(d, 10, S) + s;
    const float* q0 = Q + rows(L.m.b_v0[d], kQ, S);
    const float* q1 = Q + rows(L.m.b_v1[d], kQ, S);
    FEnt e0[2], e1[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      e0[h] = fbc_ent(k, kind, ad, val + h, S, nx, ny, q0 + h);
      e1[h] = fbc_ent(k, kind, ad, val + 5 * S + h, S, nx, ny, q1 + h);
    }
    f2 w0[4], w1[4];
    W(L.m.b_v0[d], w0);
    W(L.m.b_v1[d], w1);
    const f2 eb[4] = {add2(make_float2(e0[0].f, e0[1].f), make_float2(e1[0].f, e1[1].f)),
                      add2(make_float2(e0[0].vx, e0[1].vx), make_float2(e1[0].vx, e1[1].vx)),
                      add2(make_float2(e0[0].vy, e0[1].vy), make_float2(e1[0].vy, e1[1].vy)),
                      add2(make_float2(e0[0].l, e0[1].l), make_float2(e1[0].l, e1[1].l))};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const f2 dW = mul2(sub2(sub2(eb[i], w0[i]), w1[i]), sp(0.5f));
      dE[2 * i] = fma2(sp(nx), dW, dE[2 * i]);
      dE[2 * i + 1] = fma2(sp(ny), dW, dE[2 * i + 1]);
    }
  }
  const f2 f = sp(L.m.c_inv2a[c]);
#pragma unroll
  for (int i = 0; i < kG; ++i) dE[i] = mul2(dE[i], f);
  f2 avg[4];
  if (u < L.m.nic) {
    const f2 t3 = sp(1.0f / 3.0f);
#pragma unroll
    for (int i = 0; i < 4; ++i) avg[i] = fma2(wv[2][i], t3, fma2(wv[1][i], t3, mul2(wv[0][i], t3)));
  } else {
    float a[2][4] = {{0.0f, 0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f, 0.0f}};
    const int cnt = L.m.c_nbr_off[c + 1] - L.m.c_nbr_off[c];
    for (int j = L.m.c_nbr_off[c]; j < L.m.c_nbr_off[c + 1]; ++j) {
      const int d = L.m.c_nbr[j];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int vb = q ? L.m.bf_v1[d] : L.m.bf_v0[d];
        const float* val = L.bval + rows(d, 10, S) + (vb == L.m.b_v0[d] ? 0 : 5) * S + s;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const FEnt e = fbc_ent(k, L.m.b_kind[d], L.m.b_adiab[d], val + h, S, L.m.bf_nx[d], L.m.bf_ny[d],
                                 Q + rows(vb, kQ, S) + h);
          a[h][0] += e.f; a[h][1] += e.vx; a[h][2] += e.vy; a[h][3] += e.l;
        }
      }
    }
    const f2 sc = sp(0.5f / (float)cnt);
#pragma unroll
    for (int i = 0; i < 4; ++i) avg[i] = mul2(make_float2(a[0][i], a[1][i]), sc);
  }
  const PViscK K = pviscous_K(k, make_float2(L.mu[s], L.mu[s + 1]), avg[1], avg[2], avg[3], dE);
  float* Fo = L.Fv + rows(u, 9, S) + s;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    f2 fx, fy, fe;
    pviscous_apply(K, n[2 * q], n[2 * q + 1], fx, fy, fe);
    st2(Fo + (3 * q) * S, fx); st2(Fo + (3 * q + 1) * S, fy); st2(Fo + (3 * q + 2) * S, fe);
  }
  if (u >= L.m.nic) {
    const int d = u - L.m.nic;
    const float nbx = L.m.b_nx[d], nby = L.m.b_ny[d];
    f2 fx, fy, fe;
    pviscous_apply(K, nbx, nby, fx, fy, fe);
    if (L.m.b_adiab[d]) {   // fe - cor with cor = -(c2 e4^2 (dT/dn)) (the adiabatic wall's heat flux)
      const f2 dn = fma2(dE[7], sp(nby), mul2(dE[6], sp(nbx)));
      fe = fma2(mul2(mul2(K.c2, K.e4), K.e4), dn, fe);
    }
    float* Fb = L.Fvb + rows(d, 3, S) + s;
    st2(Fb, fx); st2(Fb + S, fy); st2(Fb + 2 * S, fe);
  }
}

// Residual gather in the fixed per-vertex edge order and the SSP-RK3 stage
// update (src/fv.cc:1635-1658), state r -> state (r+1) % 3, one vertex and H
// pairs of samples per thread.  Held or finished samples copy their state
// through.
template <int ST, int BS, bool BND, int H = kLanePairs>
__global__ void __launch_bounds__(BS) kb_gather_update(Batch B, BParams k, int r) {
  const unsigned w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const Item it = item_of_pair<ST, IT_VERTEX, H>(B, w, threadIdx.x & 31);
  if (!it.ok) return;
  const Level& L = B.lev[it.l];
  const int v = it.v, s = it.s;
  const int S = L.P;   // row pitch
  const size_t ov = rows(v, kQ, S) + s;
  const float* Q = L.Q[r] + ov;
  float* Qn = L.Q[(r + 1) % 3] + ov;
  int2 act[H];
  bool any = false;
#pragma unroll
  for (int h = 0; h < H; ++h) {
    act[h] = *reinterpret_cast<const int2*>(L.c.active + s + 2 * h);
    any = any || act[h].x || act[h].y;
  }
  if (!any) {
#pragma unroll
    for (int h = 0; h < H; ++h)
#pragma unroll
      for (int c = 0; c < kQ; ++c) st2(Qn + c * S + 2 * h, ld2(Q + c * S + 2 * h));
    return;
  }
  f2 r0[H], r1[H], r2[H], r3[H];
#pragma unroll
  for (int h = 0; h < H; ++h) r0[h] = r1[h] = r2[h] = r3[h] = sp(0.0f);
  const int j0 = L.m.ce_off[v], j1 = L.m.ce_off[v + 1];
#pragma unroll 4
  for (int j = j0; j < j1; ++j) {
    const int ent = L.m.ce_ent[j];
    const float* Fe = L.F + rows(ent >> 1, 4, S) + s;
    const f2 sg = sp((ent & 1) ? -1.0f : 1.0f);
#pragma unroll
    for (int h = 0; h < H; ++h) {
      r0[h] = fma2(ld2(Fe + 2 * h), sg, r0[h]); r1[h] = fma2(ld2(Fe + S + 2 * h), sg, r1[h]);
      r2[h] = fma2(ld2(Fe + 2 * S + 2 * h), sg, r2[h]); r3[h] = fma2(ld2(Fe + 3 * S + 2 * h), sg, r3[h]);
    }
  }
  if (BND) {   // boundary and viscous contributions in list order (src/fv.cc:1100-1188, 1197-1320)
    for (int j = L.m.cb_off[v]; j < L.m.cb_off[v + 1]; ++j) {
      const int ent = L.m.cb_ent[j];
      const int type = ent & 3, idx = ent >> 2;
      if (type == 0) {
        const float* Fe = L.Fb + rows(idx, 4, S) + s;
        const f2 hf = sp(0.5f);
#pragma unroll
        for (int h = 0; h < H; ++h) {
          r0[h] = fma2(ld2(Fe + 2 * h), hf, r0[h]); r1[h] = fma2(ld2(Fe + S + 2 * h), hf, r1[h]);
          r2[h] = fma2(ld2(Fe + 2 * S + 2 * h), hf, r2[h]); r3[h] = fma2(ld2(Fe + 3 * S + 2 * h), hf, r3[h]);
        }
      } else if ((type == 2 || type == 3) && k.model == 1) {
        const float* Fe = (type == 2 ? L.Fv : L.Fvb) + rows(idx, 3, S) + s;
        const f2 hf = sp(type == 2 ? -0.5f : 0.5f);
#pragma unroll
        for (int h = 0; h < H; ++h) {
          r1[h] = fma2(ld2(Fe + 2 * h), hf, r1[h]); r2[h] = fma2(ld2(Fe + S + 2 * h), hf, r2[h]);
          r3[h] = fma2(ld2(Fe + 2 * S + 2 * h), hf, r3[h]);
        }
      }
    }
  }
  // Shu-Osher SSP-RK3 stage (src/constants.h:4-6)
  const f2 a_rk = sp(r == 0 ? 0.0f : (r == 1 ? 0.75f : 1.0f / 3.0f));
  const f2 b_rk = sp(r == 0 ? 1.0f : (r == 1 ? 0.25f : 2.0f / 3.0f));
  const float area = L.m.area[v];
  const float* Uo = L.Uold + rows(v, 4, S) + s;
#pragma unroll
  for (int h = 0; h < H; ++h) {
    const int o = 2 * h;
    const f2 u0 = ld2(Q + o), v0 = ld2(Q + S + o), p0 = ld2(Q + 2 * S + o), V50 = ld2(Q + 4 * S + o);
    const f2 rho0 = mul2(neg2(V50), p0);
    const f2 c2 = mul2(make_float2((float)L.c.dt[s + o] / area, (float)L.c.dt[s + o + 1] / area), neg2(b_rk));
    const f2 cr = fma2(r0[h], c2, fma2(ld2(Uo + o), a_rk, mul2(rho0, b_rk)));
    const f2 cx = fma2(r1[h], c2, fma2(ld2(Uo + S + o), a_rk, mul2(mul2(rho0, u0), b_rk)));
    const f2 cy = fma2(r2[h], c2, fma2(ld2(Uo + 2 * S + o), a_rk, mul2(mul2(rho0, v0), b_rk)));
    const f2 E0 = fma2(p0, sp(k.inv_gm1), mul2(mul2(sp(0.5f), fma2(v0, v0, mul2(u0, u0))), rho0));
    const f2 cE = fma2(r3[h], c2, fma2(ld2(Uo + 3 * S + o), a_rk, mul2(E0, b_rk)));
    const f2 ir = make_float2(1.0f / cr.x, 1.0f / cr.y);
    const f2 u = mul2(cx, ir), vv = mul2(cy, ir);
    const f2 p = mul2(sp(k.gamma - 1.0f), fma2(sp(-0.5f), fma2(cy, vv, mul2(cx, u)), cE));
    const f2 hc = mul2(sp(0.5f), cr);
    const f2 beta = make_float2(hc.x / p.x, hc.y / p.y);
    const f2 sent = make_float2(__fmaf_rn(-k.gamma, logf(cr.x), logf(p.x)), __fmaf_rn(-k.gamma, logf(cr.y), logf(p.y)));
    const f2 V1 = fma2(sub2(sp(k.gamma), sent), sp(k.inv_gm1), neg2(mul2(fma2(vv, vv, mul2(u, u)), beta)));
    f2 out[kQ] = {u, vv, p, V1, mul2(sp(-2.0f), beta)};
    if (!act[h].x || !act[h].y) {   // a held sample keeps its state
#pragma unroll
      for (int c = 0; c < kQ; ++c) {
        const f2 old = ld2(Q + c * S + o);
        if (!act[h].x) out[c].x = old.x;
        if (!act[h].y) out[c].y = old.y;
      }
    }
#pragma unroll
    for (int c = 0; c < kQ; ++c) st2(Qn + c * S + o, out[c]);
    if (act[h].x && (!(p.x > 0.0f) || !(cr.x > 0.0f) || !isfinite(u.x) || !isfinite(vv.x) || !isfinite(p.x)))
      L.c.bad[s + o] = 1;
    if (act[h].y && (!(p.y > 0.0f) || !(cr.y > 0.0f) || !isfinite(u.y) || !isfinite(vv.y) || !isfinite(p.y)))
      L.c.bad[s + o + 1] = 1;
  }
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

// A uniform initial state per sample: rec[c * S + s] holds u, v, p, V1, V5 of sample s.
__global__ void kb_ic_uniform(Level L, const float* __restrict__ rec) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)L.m.nv * L.S) return;
  const int v = (int)(t / L.S), s = (int)(t % L.S);
  float* q = L.Q[0] + rows(v, kQ, L.P) + s;
#pragma unroll
  for (int c = 0; c < kQ; ++c) q[c * L.P] = rec[c * L.S + s];
}

// compute_forces (src/force.cc:116-219) of every sample of a level at its
// current state: pressure and (Navier-Stokes) viscous force on the faces of
// each force definition.  Face records (d, dq, k0, k1) as the single-solve
// tg_forces builds them (the condition of bface[f] applied, f the force
// index).  Block (force, group of 32 samples), one sample per lane, warps
// striding the faces; FP64 sums in a fixed order; out[(s nf + f) 4 + c].
// Needs the vertex gradients G of the current state.
template <int VT>
__global__ void __launch_bounds__(32 * VT) kb_forces(Level L, BParams k, const int4* __restrict__ faces,
                                                     const int* __restrict__ off, int nf, double* __restrict__ out) {
  const int lane = threadIdx.x & 31, vg = threadIdx.x >> 5;
  const int f = blockIdx.x % nf, s = (blockIdx.x / nf) * 32 + lane;
  const int S = L.P;   // row pitch
  const float* Q = L.Q[0] + s;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int j = off[f] + vg; j < off[f + 1]; j += VT) {
    const int4 rr = faces[j];
    const int d = rr.x, dq = rr.y;
    const int v0 = L.m.b_v0[d], v1 = L.m.b_v1[d];
    const float nx = L.m.b_nx[d], ny = L.m.b_ny[d];
    const float* q0 = Q + rows(v0, kQ, S);
    const float* q1 = Q + rows(v1, kQ, S);
    FPrim s0 = fprim(k, q0, S), s1 = fprim(k, q1, S);
    FEnt e0{q0[3 * S], -q0[4 * S] * q0[0], -q0[4 * S] * q0[S], q0[4 * S]};
    FEnt e1{q1[3 * S], -q1[4 * S] * q1[0], -q1[4 * S] * q1[S], q1[4 * S]};
    if (dq >= 0) {
      const int kind = L.m.b_kind[dq], ad = L.m.b_adiab[dq];
      const float qx = L.m.b_nx[dq], qy = L.m.b_ny[dq];
      const float* val0 = L.bval + rows(dq, 10, S) + 5 * rr.z * S + s;
      const float* val1 = L.bval + rows(dq, 10, S) + 5 * rr.w * S + s;
      fbc_apply1(kind, ad, val0, S, qx, qy, s0);
      fbc_apply1(kind, ad, val1, S, qx, qy, s1);
      e0 = fbc_ent(k, kind, ad, val0, S, qx, qy, q0);
      e1 = fbc_ent(k, kind, ad, val1, S, qx, qy, q1);
    }
    const double pr = 0.5 * ((double)s0.p + (double)s1.p);
    acc[0] += nx * pr;
    acc[1] += ny * pr;
    if (k.model == 1) {
      const float mu = L.mu[s];
      const float f0 = 1.0f / e0.l, f1 = 1.0f / e1.l;
      const float* G0 = L.G + rows(v0, kG, S) + s;
      const float* G1 = L.G + rows(v1, kG, S) + s;
      // u = -V2 / V5: grad u = -grad V2 / V5 + V2 grad V5 / V5^2 (src/force.cc:169-179)
      const float ux0 = G0[2 * S] * -f0 + G0[6 * S] * (f0 * e0.vx * f0), uy0 = G0[3 * S] * -f0 + G0[7 * S] * (f0 * e0.vx * f0);
      const float ux1 = G1[2 * S] * -f1 + G1[6 * S] * (f1 * e1.vx * f1), uy1 = G1[3 * S] * -f1 + G1[7 * S] * (f1 * e1.vx * f1);
      const float vx0 = G0[4 * S] * -f0 + G0[6 * S] * (f0 * e0.vy * f0), vy0 = G0[5 * S] * -f0 + G0[7 * S] * (f0 * e0.vy * f0);
      const float vx1 = G1[4 * S] * -f1 + G1[6 * S] * (f1 * e1.vy * f1), vy1 = G1[5 * S] * -f1 + G1[7 * S] * (f1 * e1.vy * f1);
      const float gux = ux0 * 0.5f + ux1 * 0.5f, guy = uy0 * 0.5f + uy1 * 0.5f;
      const float gvx = vx0 * 0.5f + vx1 * 0.5f, gvy = vy0 * 0.5f + vy1 * 0.5f;
      const float div = gux + gvy;
      const float sxx = 2.0f * mu * (gux - (1.0f / 3.0f) * div);
      const float syy = 2.0f * mu * (gvy - (1.0f / 3.0f) * div);
      const float sxy = mu * (guy + gvx);
      acc[2] += -(double)(sxx * nx + sxy * ny);
      acc[3] += -(double)(sxy * nx + syy * ny);
    }
  }
  __shared__ double red[4][VT][32];
#pragma unroll
  for (int c = 0; c < 4; ++c) red[c][vg][lane] = acc[c];
  __syncthreads();
  if (vg == 0) {
    for (int i = 1; i < VT; ++i)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[c] += red[c][i][lane];
#pragma unroll
    for (int c = 0; c < 4; ++c) out[((size_t)s * nf + f) * 4 + c] = acc[c];
  }
}

// Initial states from parameter-file expressions (InitialCondition::value,
// src/ic.h:79-104) per (vertex, sample), sample s with random numbers
// rnd[s * nrnd ..]; evaluated in FP64, stored as the FP32 record.  err: bit 8 a
// state with T <= 0 or p <= 0 (or not finite), lower bits pert errors.
__global__ void kb_ic_expr(Level L, BParams k, expr::Field5 f, const double* __restrict__ rnd, int nrnd,
                           int* __restrict__ err) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)L.m.nv * L.S) return;
  const int v = (int)(t / L.S), s = (int)(t % L.S);
  const double x = L.m.x[v], y = L.m.y[v];
  const double* row = rnd + (size_t)s * nrnd;
  int e = 0;
  const double T = expr::eval5(f, 0, x, y, 0.0, row, nrnd, &e);
  const double u = expr::eval5(f, 1, x, y, 0.0, row, nrnd, &e);
  const double vv = expr::eval5(f, 2, x, y, 0.0, row, nrnd, &e);
  const double p = expr::eval5(f, 4, x, y, 0.0, row, nrnd, &e);
  if (!(T > 0.0) || !(p > 0.0) || !isfinite(u) || !isfinite(vv) || !isfinite(T) || !isfinite(p)) e |= 8;
  if (e) { atomicOr(err, e); return; }
  const double g = (double)k.gamma;
  const double rho = p / ((double)k.R * T);
  const double beta = rho / (2.0 * p);
  const double sent = log(p) - g * log(rho);
  const double V1 = (g - sent) / (g - 1.0) - (u * u + vv * vv) * beta;
  float* q = L.Q[0] + rows(v, kQ, L.P) + s;
  q[0] = (float)u;
  q[L.P] = (float)vv;
  q[2 * L.P] = (float)p;
  q[3 * L.P] = (float)V1;
  q[4 * L.P] = (float)(-2.0 * beta);
}

// Per-sample boundary values of the faces of one boundary tag from expressions
// (BoundaryCondition at each face vertex, time t): variable c of the record
// (T, u, v, w, p) is written where bit c of mask is set.
__global__ void kb_bc_expr(Level L, expr::Field5 f, int mask, const int* __restrict__ btag, int tag,
                           const double* __restrict__ rnd, int nrnd, double t, int* __restrict__ err) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= 2LL * L.m.nb * L.S) return;
  const int slot = (int)(i / L.S), s = (int)(i % L.S);
  const int d = slot >> 1, q = slot & 1;
  if (btag[d] != tag) return;
  const int vtx = q ? L.m.b_v1[d] : L.m.b_v0[d];
  const double x = L.m.x[vtx], y = L.m.y[vtx];
  const double* row = rnd + (size_t)s * nrnd;
  int e = 0;
  float* val = L.bval + rows(d, 10, L.P) + 5 * q * L.P + s;
  for (int c = 0; c < 5; ++c)
    if ((mask >> c) & 1) val[c * L.P] = (float)expr::eval5(f, c, x, y, t, row, nrnd, &e);
  if (e) atomicOr(err, e);
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
