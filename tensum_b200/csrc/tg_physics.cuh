// tg_physics.cuh -- pointwise and edgewise physics of the TENSUM hot path, 2D.
//
// Device restatement of Material (src/material.h, src/material.cc) and the
// numerical fluxes (src/kep*.cc, src/roe_ec.cc, src/simple_avg.cc).  The
// reference carries z components that are identically zero in 2D
// (n_z = 0, w = 0); they are dropped here, which leaves every value unchanged
// (only exact +-0 terms disappear).  Operand order follows the reference so
// that results differ from it only by FMA contraction and the last-ulp
// behaviour of log/sqrt.
//
// Variable order on the device:
//   primitive  P = (T, u, v, p)
//   conserved  U = (rho, rho u, rho v, E)
//   entropy    W = (V1, V2, V3, V5)  (reference EntVar entf, entv.x, entv.y, entl)
//   flux / residual = (mass, x-momentum, y-momentum, energy)
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace tg {

enum : int { FLUX_TECNO_ROE = 0, FLUX_TECNO_RUSANOV = 1, FLUX_KEPEC = 2, FLUX_ROE_EC = 3, FLUX_KEP = 4, FLUX_AVG = 5 };
enum : int { RECON_FIRST = 0, RECON_SECOND = 1, RECON_SECOND_MUSCL = 2, RECON_VAN_ALBADA = 3,
             RECON_TVD_MINMOD = 4, RECON_TVB_MINMOD = 5, RECON_ENO2 = 6 };
enum : int { BC_NONE = 0, BC_SLIP = 1, BC_NOSLIP = 2, BC_FARFIELD = 3, BC_INLET = 4, BC_OUTLET = 5,
             BC_PRESSURE = 6, BC_PERIODIC = 7 };

struct Params {
  double gamma, R, Cp, prandtl;
  double sqrt_gm1, inv_gamma, inv_gm1;   // sqrt(gamma - 1), 1/gamma, 1/(gamma - 1)
  double gp1_gm1;                        // (gamma + 1)/(gamma - 1)
  double mu_ref, T0, Tref, omega;
  double ev_alpha, ev_beta, tvbM;
  double cfl;
  int model;      // 0 euler, 1 ns
  int flux, mu_model, recon;
  int nd, visc, heat;
  int liou;       // Liou's carbuncle switch active (liou_fix with kepes_tecno_roe)
  int strong;     // bc_scheme strong
  int fuse_dt;    // the last stage's update also forms the next step's local dt and U_old
  int axi;        // axisymmetric: residual contributions and the update weighted by radii
};

struct Prim { double T, u, v, p; };
struct Cons { double r, mx, my, E; };
struct Ent { double f, vx, vy, l; };
struct Flx { double m, x, y, e; };

__device__ __forceinline__ double dmin_(double a, double b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ double dmax_(double a, double b) { return (a < b) ? b : a; }  // std::max

// Ismail-Roe logarithmic mean (a - b)/ln(a/b), src/material.h:24-42: returns
// F with logmean = 0.5 (a + b) / F.  The reference forms f = (xi - 1)/(xi + 1)
// from xi = b/a; f = (b - a)/(b + a) is the same quantity with one division
// instead of two (and no cancellation in xi - 1), and the series divides by
// 3, 5, 7 where multiplying by the reciprocals differs by at most an ulp.
__device__ __forceinline__ double logavg_F(double a, double b) {
  double f = (b - a) / (b + a);
  double u = f * f;
  if (u < 1.0e-2) {
    double u2 = u * u;
    double u3 = u2 * u;
    return 1.0 + u * (1.0 / 3.0) + u2 * (1.0 / 5.0) + u3 * (1.0 / 7.0);
  }
  return log(b / a) / 2.0 / f;
}

__device__ __forceinline__ double logavg(double a, double b) { return 0.5 * (a + b) / logavg_F(a, b); }
// 1 / logavg(a, b), for the callers that only ever divide by the log mean
__device__ __forceinline__ double inv_logavg(double a, double b) { return logavg_F(a, b) / (0.5 * (a + b)); }

__device__ __forceinline__ double density(const Params& k, const Prim& q) { return q.p / (k.R * q.T); }
__device__ __forceinline__ double sound_speed(const Params& k, const Prim& q) { return sqrt(k.gamma * k.R * q.T); }
__device__ __forceinline__ double entropy_fn(const Params& k, const Prim& q) {
  return log(q.p) - k.gamma * log(density(k, q));
}

__device__ __forceinline__ double viscosity(const Params& k, double T) {   // src/material.h:551-568
  if (k.mu_model == 1) return k.mu_ref * pow(T, 1.5) / (T + k.T0);
  if (k.mu_model == 2) return k.mu_ref * pow(T / k.Tref, k.omega);
  return k.mu_ref;
}

// The energy's multiply-adds are written out so that every kernel that forms
// U_old from a state (the first stage's pass, or the previous step's last
// update) rounds it the same way.
__device__ __forceinline__ Cons prim2con(const Params& k, const Prim& q) {   // src/material.h:501-513
  Cons c;
  double rho = density(k, q);
  c.r = rho;
  c.mx = q.u * rho;
  c.my = q.v * rho;
  c.E = fma(0.5 * fma(q.u, q.u, q.v * q.v), rho, q.p / (k.gamma - 1.0));
  return c;
}

__device__ __forceinline__ Prim con2prim(const Params& k, const Cons& c) {   // src/material.h:518-529
  Prim q;
  double ir = 1.0 / c.r;
  q.u = c.mx * ir;
  q.v = c.my * ir;
  q.p = (k.gamma - 1.0) * (c.E - 0.5 * (c.mx * c.mx + c.my * c.my) / c.r);
  q.T = q.p / (k.R * c.r);
  return q;
}

// V5 = -2 beta of prim2ent alone, with its operations (no logarithm).
__device__ __forceinline__ double prim2ent_v5(const Params& k, const Prim& q) {
  double beta = density(k, q) / (2 * q.p);
  return -2 * beta;
}

__device__ __forceinline__ Ent prim2ent(const Params& k, const Prim& q) {   // src/material.h:534-546
  Ent e;
  double rho = density(k, q);
  double beta = rho / (2 * q.p);
  double s = entropy_fn(k, q);
  e.f = (k.gamma - s) / (k.gamma - 1) - (q.u * q.u + q.v * q.v) * beta;
  e.vx = q.u * (2 * beta);
  e.vy = q.v * (2 * beta);
  e.l = -2 * beta;
  return e;
}

// ----------------------------------------------------------------- limiters
__device__ __forceinline__ double minmod_tvd(double a, double b) {          // src/limiter.h:14-27
  if (a < 0.0 && b < 0.0) return -dmin_(-a, -b);
  if (a > 0.0 && b > 0.0) return dmin_(a, b);
  return 0.0;
}

template <int RECON>
__device__ __forceinline__ double limited_slope(double ul, double ur, double h, double M) {  // src/reconstruct.cc:101-134
  if (RECON == RECON_VAN_ALBADA) {
    double s = dmax_(0.0, (2 * ul * ur + 1.0e-14) / (ul * ul + ur * ur + 1.0e-14));
    return 0.25 * s * ((1.0 - (1.0 / 3.0) * s) * ul + (1.0 + (1.0 / 3.0) * s) * ur);
  } else if (RECON == RECON_TVD_MINMOD) {
    return 0.5 * minmod_tvd(ul, ur);
  } else if (RECON == RECON_ENO2) {
    return 0.5 * ((fabs(ul) < fabs(ur)) ? ul : ur);
  } else {  // TVB minmod, src/limiter.h:66-77
    double c = 0.5 * (ul + ur);
    if (fabs(c) < M * (h * h)) return 0.5 * c;
    return 0.5 * minmod_tvd(ul, ur);
  }
}

// Jump Z_ji - Z_ij of Material::reconstruct (src/reconstruct.cc:139-188) for
// one component, from the first-order jump d = Z_r - Z_l and the slopes.
template <int RECON>
__device__ __forceinline__ double reconstructed_jump(double d, double gl, double gr, double h, double M) {
  if (RECON == RECON_FIRST) {
    return d;
  } else if (RECON == RECON_SECOND) {
    return d - 0.5 * gr - 0.5 * gl;
  } else if (RECON == RECON_SECOND_MUSCL) {
    const double K = 1.0 / 3.0;
    double sl = ((2.0 * gl - d) * (1.0 - K) + d * (1.0 + K)) * 0.25;
    double sr = ((2.0 * gr - d) * (1.0 - K) + d * (1.0 + K)) * 0.25;
    return d - sr - sl;
  } else {
    return d - limited_slope<RECON>(2.0 * gr - d, d, h, M) - limited_slope<RECON>(2.0 * gl - d, d, h, M);
  }
}

// Whether reconstructed_jump<RECON> is positively homogeneous of degree one in
// (d, gl, gr): van Albada's 1e-14 regularisation and the TVB threshold M h^2
// carry their own scale.
template <int RECON>
__host__ __device__ constexpr bool recon_homogeneous() {
  return RECON != RECON_VAN_ALBADA && RECON != RECON_TVB_MINMOD;
}

// Material::reconstruct (src/reconstruct.cc:139-188) for one component.
template <int RECON>
__device__ __forceinline__ void reconstruct1(double l, double r, double gl, double gr, double h, double M,
                                             double& rl, double& rr) {
  if (RECON == RECON_FIRST) {
    rl = l; rr = r;
  } else if (RECON == RECON_SECOND) {
    rl = l + 0.5 * gl;
    rr = r - 0.5 * gr;
  } else if (RECON == RECON_SECOND_MUSCL) {
    const double K = 1.0 / 3.0;
    double d = r - l;
    double dl = 2.0 * gl - d;
    rl = l + (dl * (1.0 - K) + d * (1.0 + K)) * 0.25;
    double dr = 2.0 * gr - d;
    rr = r - (dr * (1.0 - K) + d * (1.0 + K)) * 0.25;
  } else {
    double d = r - l;
    double dl = 2.0 * gl - d;
    rl = l + limited_slope<RECON>(dl, d, h, M);
    double dr = 2.0 * gr - d;
    rr = r - limited_slope<RECON>(dr, d, h, M);
  }
}

// ------------------------------------------------------------------- fluxes
// Per-vertex quantities every flux reads.  The reference recomputes them for
// each edge from the primitive state (Density, beta = 0.5/(R T), Entropy,
// sound_speed ...); evaluating them once per vertex with the same expressions
// gives the same values.
struct VRec {
  double rho;   // p / (R T)                                    src/material.h:596
  double u, v, p;
  double beta;  // 0.5 / (R T)                                  src/kepec.cc:23
  double V1;    // (gamma - s)/(gamma - 1) - beta |u|^2, s = ln p - gamma ln rho   src/kepes_tecno_roe.cc:100-104
  double a;     // sqrt(gamma R T)                              src/material.h:587
  double b;     // sqrt(rho / p)                                src/roe_ec.cc:22
};

template <int FLUX>
__device__ __forceinline__ VRec make_vrec(const Params& k, const Prim& q) {
  VRec r;
  r.rho = q.p / (k.R * q.T);
  r.u = q.u;
  r.v = q.v;
  r.p = q.p;
  r.beta = 0.5 / (k.R * q.T);
  r.V1 = 0.0;
  r.a = 0.0;
  r.b = 0.0;
  if (FLUX == FLUX_TECNO_ROE || FLUX == FLUX_TECNO_RUSANOV) {
    double s = log(q.p) - k.gamma * log(r.rho);
    r.V1 = (k.gamma - s) / (k.gamma - 1.0) - r.beta * (q.u * q.u + q.v * q.v);
  }
  if (FLUX == FLUX_TECNO_ROE || FLUX == FLUX_KEP) r.a = sqrt(k.gamma * k.R * q.T);
  if (FLUX == FLUX_ROE_EC) r.b = sqrt(r.rho / q.p);
  return r;
}

// The same record from the stored entropy variables: V5 = -2 beta gives
// beta = -V5/2 and rho = 2 beta p = -V5 p, and V1 is the stored first entropy
// variable, so no division or logarithm is needed per vertex.  The stored
// variables come from prim2ent (beta = rho/(2p), src/material.h:534-546), the
// flux recomputes them from (T, p) (beta = 0.5/(R T)); the two differ in the
// last ulp only.
template <int FLUX>
__device__ __forceinline__ VRec make_vrec_w(const Params& k, double u, double v, double p, double T, double V1,
                                            double V5) {
  VRec r;
  r.rho = -V5 * p;
  r.u = u;
  r.v = v;
  r.p = p;
  r.beta = -0.5 * V5;
  r.V1 = V1;
  r.a = 0.0;
  r.b = 0.0;
  if (FLUX == FLUX_TECNO_ROE || FLUX == FLUX_KEP) r.a = sqrt(k.gamma * k.R * T);
  if (FLUX == FLUX_ROE_EC) r.b = sqrt(-V5);
  return r;
}

// The averages the KEPEC and TeCNO fluxes share: the density log mean, the
// inverse of the beta log mean and p = (rho_l + rho_r) / (2 (beta_l + beta_r)),
// from two reciprocals and one division instead of five divisions: the
// beta sum's reciprocal serves beta's log-mean ratio f, 1/beta_ln and p.
__device__ __forceinline__ double logavg_F_of(double f, double a, double b) {
  double u = f * f;
  if (u < 1.0e-2) {
    double u2 = u * u;
    double u3 = u2 * u;
    return 1.0 + u * (1.0 / 3.0) + u2 * (1.0 / 5.0) + u3 * (1.0 / 7.0);
  }
  return log(b / a) / 2.0 / f;
}
__device__ __forceinline__ void shared_means(const VRec& L, const VRec& R, double& rho, double& ibeta, double& p) {
  const double sr = L.rho + R.rho, sb = L.beta + R.beta;
  const double isr = 1.0 / sr, isb = 1.0 / sb;
  rho = 0.5 * sr / logavg_F_of((R.rho - L.rho) * isr, L.rho, R.rho);
  ibeta = logavg_F_of((R.beta - L.beta) * isb, L.beta, R.beta) * (2.0 * isb);
  p = 0.5 * sr * isb;
}

__device__ __forceinline__ Flx kepec_flux(const Params& k, const VRec& L, const VRec& R, double unx, double uny) {
  // src/kepec.cc:10-38; 1/((gamma-1) beta_ln) is formed from 1/beta_ln directly
  double rho, ibeta, p;
  shared_means(L, R, rho, ibeta, p);
  double vel2 = 0.5 * ((L.u * L.u + L.v * L.v) + (R.u * R.u + R.v * R.v));
  double vx = L.u * 0.5 + R.u * 0.5, vy = L.v * 0.5 + R.v * 0.5;
  double vn = vx * unx + vy * uny;
  Flx F;
  F.m = rho * vn;
  F.x = unx * p + vx * F.m;
  F.y = uny * p + vy * F.m;
  F.e = 0.5 * (ibeta * k.inv_gm1 - vel2) * F.m + (F.x * vx + F.y * vy);
  return F;
}

__device__ __forceinline__ Flx kep_flux(const Params& k, const VRec& L, const VRec& R, double unx, double uny) {
  // src/kep.cc:10-38 (pow(a, 2.0) is the square a*a; a^2 / (gamma - 1) as a^2 times 1/(gamma - 1))
  double Hl = L.a * L.a * k.inv_gm1 + 0.5 * (L.u * L.u + L.v * L.v);
  double Hr = R.a * R.a * k.inv_gm1 + 0.5 * (R.u * R.u + R.v * R.v);
  double p = 0.5 * (L.p + R.p);
  double rho = 0.5 * (L.rho + R.rho);
  double H = 0.5 * (Hl + Hr);
  double vx = L.u * 0.5 + R.u * 0.5, vy = L.v * 0.5 + R.v * 0.5;
  double vn = vx * unx + vy * uny;
  Flx F;
  F.m = rho * vn;
  F.x = unx * p + vx * F.m;
  F.y = uny * p + vy * F.m;
  F.e = rho * H * vn;
  return F;
}

__device__ __forceinline__ Flx roe_ec_flux(const Params& k, const VRec& L, const VRec& R, double unx, double uny) {
  // src/roe_ec.cc:10-44.  The reference divides nine times per edge; here the
  // reciprocal of z1b = (b_l + b_r)/2 serves its log-mean ratio, 1/z1_ln = F_1 / z1b and
  // the three divisions by z1b, the reciprocal of the z5 sum its ratio, and
  // (gamma + 1)/(gamma - 1) is a constant: two reciprocals and one division.
  double pl = L.p, pr = R.p;
  double bl = L.b, br = R.b;
  double z1b = 0.5 * (bl + br);
  double zx = L.u * (0.5 * bl) + R.u * (0.5 * br);
  double zy = L.v * (0.5 * bl) + R.v * (0.5 * br);
  double z5l_ = bl * pl, z5r_ = br * pr;
  double z5b = 0.5 * (z5l_ + z5r_);
  double zn = zx * unx + zy * uny;
  const double i1b = 1.0 / z1b, i5s = 1.0 / (z5l_ + z5r_);
  const double F1 = logavg_F_of((br - bl) * (0.5 * i1b), bl, br);    // z1_ln = z1b / F1
  const double F5 = logavg_F_of((z5r_ - z5l_) * i5s, z5l_, z5r_);
  double z5l = z5b / F5;
  Flx F;
  F.m = z5l * zn;
  double c1 = z5b * i1b, c2 = F.m * i1b;
  F.x = unx * c1 + zx * c2;
  F.y = uny * c1 + zy * c2;
  F.e = 0.5 * (k.gp1_gm1 * F.m * (F1 * i1b) + (F.x * zx + F.y * zy)) * i1b;
  return F;
}

__device__ __forceinline__ Flx avg_flux(const Params& k, const VRec& L, const VRec& R, double unx, double uny) {
  // src/simple_avg.cc:10-46
  double El = 0.5 * L.rho * (L.u * L.u + L.v * L.v) + L.p / (k.gamma - 1);
  double Er = 0.5 * R.rho * (R.u * R.u + R.v * R.v) + R.p / (k.gamma - 1);
  double vnl = L.u * unx + L.v * uny, vnr = R.u * unx + R.v * uny;
  double ml = L.rho * vnl, mr = R.rho * vnr;
  Flx F;
  F.m = 0.0 + ml * 0.5;
  F.m += mr * 0.5;
  F.x = 0.0 + (unx * L.p + L.u * ml) * 0.5;
  F.x += (unx * R.p + R.u * mr) * 0.5;
  F.y = 0.0 + (uny * L.p + L.v * ml) * 0.5;
  F.y += (uny * R.p + R.v * mr) * 0.5;
  F.e = 0.0 + ((El + L.p) * vnl) * 0.5;
  F.e += ((Er + R.p) * vnr) * 0.5;
  return F;
}

// KEPES-TeCNO (src/kepes_tecno_roe.cc:11-173, src/kepes_tecno_rusanov.cc:11-164):
// KEPEC central flux minus 0.5 R Lambda (Z_ji - Z_ij), Z = R^T V reconstructed
// along the edge with the slopes R^T (grad V . dr).  dEl/dEr are the entropy-
// variable gradients (V1,V2,V3,V5) x (x,y) at the two vertices, (dx,dy) the
// edge vector x_r - x_l.
template <int ROE, int RECON>
__device__ __forceinline__ Flx tecno_flux(const Params& k, const VRec& L, const VRec& Rp, double unx, double uny,
                                          double dx, double dy, const double* dEl, const double* dEr, int ssw = 0) {
  const double g = k.gamma;
  double rho, ibeta, p;                          // rho_ln, 1 / beta_ln, p
  shared_means(L, Rp, rho, ibeta, p);
  double a = sqrt(0.5 * g * ibeta);
  double vx = L.u * 0.5 + Rp.u * 0.5, vy = L.v * 0.5 + Rp.v * 0.5;
  double vn = vx * unx + vy * uny;
  // central KEPEC part (src/kepec.cc:25-34) from the log means computed above
  Flx F;
  {
    double vel2 = 0.5 * ((L.u * L.u + L.v * L.v) + (Rp.u * Rp.u + Rp.v * Rp.v));
    F.m = rho * vn;
    F.x = unx * p + vx * F.m;
    F.y = uny * p + vy * F.m;
    F.e = 0.5 * (ibeta * k.inv_gm1 - vel2) * F.m + (F.x * vx + F.y * vy);
  }
  if (!k.nd) return F;

  double vsq = vx * vx + vy * vy;
  double v1 = vx * uny - vy * unx;
  if (recon_homogeneous<RECON>()) {
    // The reconstructions whose limiter is positively homogeneous of degree one
    // (phi(s x, s y) = s phi(x, y) for s > 0: first, second, MUSCL, minmod, ENO2)
    // commute with the scaling S of the eigenvectors: the dissipation
    // S (Lambda jump(S R0^T V)) equals S^2 (Lambda jump(R0^T V)) with
    // S0^2 = rho/(2 gamma), S1^2 = (gamma - 1) rho/gamma, S2^2 = p.  The
    // unscaled form needs one square root per edge (a) instead of three.
    const double aa = 0.5 * g * ibeta;            // a^2
    const double H2 = aa * k.inv_gm1 + 0.5 * vsq;
    auto RT0 = [&](const double* x, double* z) {
      double A = x[0] + vx * x[1] + vy * x[2];
      double B = unx * x[1] + uny * x[2] + vn * x[3];
      double C = A + H2 * x[3];
      z[0] = C - a * B;
      z[1] = A + (0.5 * vsq) * x[3];
      z[2] = uny * x[1] - unx * x[2] + v1 * x[3];
      z[3] = C + a * B;
    };
    double Lam[4];
    if (ROE) {
      double vnl = L.u * unx + L.v * uny, vnr = Rp.u * unx + Rp.v * uny;
      double l2 = fabs(vn);
      Lam[0] = (1 + k.ev_beta) * fabs(vn - a) + k.ev_alpha * fabs((vnl - L.a) - (vnr - Rp.a));
      Lam[1] = l2;
      Lam[2] = ssw > 0 ? dmax_(l2, a) : l2;
      Lam[3] = (1 + k.ev_beta) * fabs(vn + a) + k.ev_alpha * fabs((vnl + L.a) - (vnr + Rp.a));
    } else {
      double lr = fabs(vn) + a;                  // a >= 0
      Lam[0] = Lam[1] = Lam[2] = Lam[3] = lr;
    }
    double dV[4] = {Rp.V1 - L.V1, 2 * Rp.u * Rp.beta - 2 * L.u * L.beta, 2 * Rp.v * Rp.beta - 2 * L.v * L.beta,
                    -2 * Rp.beta - -2 * L.beta};
    double gl[4], gr[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      gl[i] = dEl[2 * i] * dx + dEl[2 * i + 1] * dy;
      gr[i] = dEr[2 * i] * dx + dEr[2 * i + 1] * dy;
    }
    double d[4], sgl[4], sgr[4];
    RT0(dV, d);
    RT0(gl, sgl);
    RT0(gr, sgr);
    double q[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) q[i] = Lam[i] * reconstructed_jump<RECON>(d[i], sgl[i], sgr[i], 0.0, 0.0);
    const double s01 = rho * k.inv_gamma;
    q[0] *= 0.5 * s01; q[1] *= (g - 1.0) * s01; q[2] *= p; q[3] *= 0.5 * s01;
    double sum = q[0] + q[1] + q[3], dif = q[3] - q[0];
    F.m -= 0.5 * sum;
    F.x -= 0.5 * (vx * sum + a * unx * dif + uny * q[2]);
    F.y -= 0.5 * (vy * sum + a * uny * dif - unx * q[2]);
    F.e -= 0.5 * (H2 * (q[0] + q[3]) + a * vn * dif + (0.5 * vsq) * q[1] + v1 * q[2]);
    return F;
  }
  // van Albada and TVB minmod: the scaled form of the reference
  double H = a * a / (g - 1.0) + 0.5 * vsq;
  double const1 = sqrt(rho * k.inv_gamma);
  double psqrt = sqrt(p);
  double S0 = sqrt(0.5) * const1, S1 = k.sqrt_gm1 * const1, S2 = psqrt;
  // The scaled eigenvector matrix (src/kepes_tecno_roe.cc:61-77) has the columns
  //   (u-a): S0 (1, vx - a nx, vy - a ny, H - a vn)   (entropy): S1 (1, vx, vy, |v|^2/2)
  //   (shear): S2 (0, ny, -nx, v1)                    (u+a): S0 (1, vx + a nx, vy + a ny, H + a vn)
  // and is applied through that structure below instead of being stored.
  auto RT = [&](const double* x, double* z) {
    double A = x[0] + vx * x[1] + vy * x[2];
    double B = unx * x[1] + uny * x[2] + vn * x[3];
    double C = A + H * x[3];
    z[0] = S0 * (C - a * B);
    z[1] = S1 * (A + (0.5 * vsq) * x[3]);
    z[2] = S2 * (uny * x[1] - unx * x[2] + v1 * x[3]);
    z[3] = S0 * (C + a * B);
  };
  double Lam[4];
  if (ROE) {
    double vnl = L.u * unx + L.v * uny, vnr = Rp.u * unx + Rp.v * uny;
    double l2 = fabs(vn);
    Lam[0] = (1 + k.ev_beta) * fabs(vn - a) + k.ev_alpha * fabs((vnl - L.a) - (vnr - Rp.a));
    Lam[1] = l2;
    Lam[2] = ssw > 0 ? dmax_(l2, a) : l2;   // Liou's modification (src/kepes_tecno_roe.cc:85-87)
    Lam[3] = (1 + k.ev_beta) * fabs(vn + a) + k.ev_alpha * fabs((vnl + L.a) - (vnr + Rp.a));
  } else {
    double lr = fabs(vn) + fabs(a);
    Lam[0] = Lam[1] = Lam[2] = Lam[3] = lr;
  }
  // Every reconstruction reads Z_l, Z_r only through Z_r - Z_l (src/reconstruct.cc:31-96),
  // so the jump is formed as R^T (V_r - V_l) with one product instead of two.
  double dV[4] = {Rp.V1 - L.V1, 2 * Rp.u * Rp.beta - 2 * L.u * L.beta, 2 * Rp.v * Rp.beta - 2 * L.v * L.beta,
                  -2 * Rp.beta - -2 * L.beta};
  double h = (RECON == RECON_TVB_MINMOD) ? sqrt(dx * dx + dy * dy) : 0.0;
  double gl[4], gr[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    gl[i] = dEl[2 * i] * dx + dEl[2 * i + 1] * dy;
    gr[i] = dEr[2 * i] * dx + dEr[2 * i + 1] * dy;
  }
  double d[4], sgl[4], sgr[4];
  RT(dV, d);
  RT(gl, sgl);
  RT(gr, sgr);
  // q = S (Lambda dZ); Diff = R Lambda dZ from the columns above
  double q[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) q[i] = Lam[i] * reconstructed_jump<RECON>(d[i], sgl[i], sgr[i], h, k.tvbM);
  q[0] *= S0; q[1] *= S1; q[2] *= S2; q[3] *= S0;
  double sum = q[0] + q[1] + q[3], dif = q[3] - q[0];
  F.m -= 0.5 * sum;
  F.x -= 0.5 * (vx * sum + a * unx * dif + uny * q[2]);
  F.y -= 0.5 * (vy * sum + a * uny * dif - unx * q[2]);
  F.e -= 0.5 * (H * (q[0] + q[3]) + a * vn * dif + (0.5 * vsq) * q[1] + v1 * q[2]);
  return F;
}

// Material::num_flux (src/material.cc:27-74) given the unit normal and |n|
// (area = |n|, unit normal = n * (1/area), as the fluxes compute them).
template <int FLUX, int RECON>
__device__ __forceinline__ Flx num_flux_unit(const Params& k, const VRec& L, const VRec& R, double unx, double uny,
                                             double area, double dx, double dy, const double* dEl, const double* dEr,
                                             int ssw = 0) {
  Flx F;
  if (FLUX == FLUX_TECNO_ROE) F = tecno_flux<1, RECON>(k, L, R, unx, uny, dx, dy, dEl, dEr, ssw);
  else if (FLUX == FLUX_TECNO_RUSANOV) F = tecno_flux<0, RECON>(k, L, R, unx, uny, dx, dy, dEl, dEr);
  else if (FLUX == FLUX_KEPEC) F = kepec_flux(k, L, R, unx, uny);
  else if (FLUX == FLUX_KEP) F = kep_flux(k, L, R, unx, uny);
  else if (FLUX == FLUX_ROE_EC) F = roe_ec_flux(k, L, R, unx, uny);
  else F = avg_flux(k, L, R, unx, uny);
  F.m *= area; F.x *= area; F.y *= area; F.e *= area;
  return F;
}

template <int FLUX, int RECON>
__device__ __forceinline__ Flx num_flux(const Params& k, const VRec& L, const VRec& R, double nx, double ny, double dx,
                                        double dy, const double* dEl, const double* dEr) {
  double area = sqrt(nx * nx + ny * ny);
  double ia = 1.0 / area;
  return num_flux_unit<FLUX, RECON>(k, L, R, nx * ia, ny * ia, area, dx, dy, dEl, dEr);
}

// Material::inviscid_bflux (src/material.cc:110-127).
__device__ __forceinline__ Flx inviscid_bflux(const Params& k, const Prim& q, const Prim& qb, double nx, double ny) {
  double vnb = qb.u * nx + qb.v * ny;
  double vn = q.u * nx + q.v * ny;
  double rho = density(k, q);
  Flx F;
  F.m = rho * vnb;
  F.x = nx * qb.p + q.u * F.m;
  F.y = ny * qb.p + q.v * F.m;
  F.e = (0.5 * rho * (q.u * q.u + q.v * q.v) + k.gamma * q.p / (k.gamma - 1.0)) * vnb + (qb.p - q.p) * vn;
  return F;
}

// Viscous matrices K_ij dV_j (src/material.cc:158-230); dE is the cell
// gradient (V1,V2,V3,V5) x (x,y).  Returns the four (x,y) flux-direction
// products needed for any normal, and e4 = 1/V5, c2 = k/R.
struct ViscK { double a1, a2, a4, b1, b2, b4, e4, c2; };

__device__ __forceinline__ ViscK viscous_K(const Params& k, const Ent& st, const double* dE) {
  double mu = viscosity(k, -1 / (k.R * st.l));
  double kk = mu * k.Cp / k.prandtl;
  if (!k.visc) mu = 0.0;
  if (!k.heat) kk = 0.0;
  double e1 = st.vx / st.l, e2 = st.vy / st.l, e4 = 1.0 / st.l;
  double c1 = 4.0 * mu / 3.0, c2 = kk / k.R, c3 = 2 * mu / 3.0;
  // dE index: V1:(0,1) V2:(2,3) V3:(4,5) V5:(6,7)
  double d1x = dE[2], d1y = dE[3], d2x = dE[4], d2y = dE[5], d4x = dE[6], d4y = dE[7];
  double K11_1 = c1 * (-d1x + e1 * d4x);
  double K11_2 = mu * (-d2x + e2 * d4x);
  double K11_4 = c1 * e1 * d1x + mu * (e2 * d2x) + (-c1 * e1 * e1 - mu * (e2 * e2) + c2 * e4) * d4x;
  double K12_1 = c3 * (d2y - e2 * d4y);
  double K12_2 = mu * (-d1y + e1 * d4y);
  double K12_4 = mu * e2 * d1y - c3 * e1 * d2y - (mu - c3) * e1 * e2 * d4y;
  double K21_1 = mu * (-d2x + e2 * d4x);
  double K21_2 = c3 * (d1x - e1 * d4x);
  double K21_4 = -c3 * e2 * d1x + mu * e1 * d2x - (mu - c3) * e1 * e2 * d4x;
  double K22_1 = mu * (-d1y + e1 * d4y);
  double K22_2 = c1 * (-d2y + e2 * d4y);
  double K22_4 = mu * (e1 * d1y) + c1 * e2 * d2y + (-mu * (e1 * e1) - c1 * e2 * e2 + c2 * e4) * d4y;
  ViscK r;
  r.a1 = K11_1 + K12_1; r.a2 = K11_2 + K12_2; r.a4 = K11_4 + K12_4;
  r.b1 = K21_1 + K22_1; r.b2 = K21_2 + K22_2; r.b4 = K21_4 + K22_4;
  r.e4 = e4;
  r.c2 = c2;
  return r;
}

__device__ __forceinline__ Flx viscous_apply(const ViscK& K, double nx, double ny) {
  Flx F;
  F.m = 0.0;
  F.x = -(K.a1 * nx + K.b1 * ny) * K.e4;
  F.y = -(K.a2 * nx + K.b2 * ny) * K.e4;
  F.e = -(K.a4 * nx + K.b4 * ny) * K.e4;
  return F;
}

// BoundaryCondition::apply, two-state form (src/bc.h:568-610).
__device__ __forceinline__ void bc_apply2(int kind, int adiabatic, const double* val, double nx, double ny,
                                          Prim& s0, Prim& s1) {
  switch (kind) {
    case BC_SLIP: {
      double meas = sqrt(nx * nx + ny * ny);
      double ux = nx * (1.0 / meas), uy = ny * (1.0 / meas);
      double fact = s0.u * ux + s0.v * uy;
      s0.u += ux * -fact;
      s0.v += uy * -fact;
      s1 = s0;
      break;
    }
    case BC_NOSLIP:
      s0.u = val[1]; s0.v = val[2];
      s1.u = s0.u; s1.v = s0.v;
      s1.p = s0.p;
      if (adiabatic) s1.T = s0.T;
      else { s0.T = val[0]; s1.T = val[0]; }
      break;
    case BC_PRESSURE: s1.p = val[4]; break;
    case BC_INLET:
      s0.T = val[0]; s0.u = val[1]; s0.v = val[2]; s0.p = val[4];
      s1 = s0;
      break;
    case BC_OUTLET: s1 = s0; break;
    case BC_FARFIELD:
      s1.T = val[0]; s1.u = val[1]; s1.v = val[2]; s1.p = val[4];
      break;
    default: break;
  }
}

// BoundaryCondition::apply, single-state form (src/bc.h:615-654).
__device__ __forceinline__ void bc_apply1(int kind, int adiabatic, const double* val, double nx, double ny, Prim& s) {
  switch (kind) {
    case BC_SLIP: {
      double meas = sqrt(nx * nx + ny * ny);
      double ux = nx * (1.0 / meas), uy = ny * (1.0 / meas);
      double fact = s.u * ux + s.v * uy;
      s.u += ux * -fact;
      s.v += uy * -fact;
      break;
    }
    case BC_NOSLIP:
      s.u = val[1]; s.v = val[2];
      if (!adiabatic) s.T = val[0];
      break;
    case BC_PRESSURE: s.p = val[4]; break;
    case BC_INLET: s.T = val[0]; s.u = val[1]; s.v = val[2]; s.p = val[4]; break;
    default: break;
  }
}

}  // namespace tg
