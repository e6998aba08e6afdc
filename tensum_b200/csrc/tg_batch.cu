// tg_batch.cu -- C ABI of the batched FP32 Monte Carlo ensembles (tensum_gpu.h,
// "batched ensembles").
//
// A batch holds one or more levels (a mesh and its samples); every level
// advances in the same launches.  One time step of the whole batch is
// captured once into a CUDA graph and replayed; the launch shape (sample tile
// and block size of the flux and gradient kernels) is chosen by tg_batch_tune.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/tensum_gpu.h"
#include "tg_batch.cuh"
#include "tg_mesh.h"

using namespace tg;
using namespace tg::batch;

namespace {

thread_local std::string g_batch_error;

struct LevelHost {
  HostLayout L;
  int S = 0;
  std::vector<void*> allocs;
};

struct Shape {
  int st, bs;
};
const Shape kShapes[] = {{32, 256}, {32, 128}, {16, 256}, {16, 128}};

}  // namespace

struct tg_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  int nlev = 0;
  LevelHost lh[kMaxLevels];
  Batch B{};
  BParams prm{};
  int* stop = nullptr;           // device stop counter (read by kb_step_begin)
  double* tinst = nullptr;
  int shape = 0;                 // index into kShapes
  bool bnd = false;              // walls / far field or Navier-Stokes: the boundary and viscous passes run
  int dt_chunks = 1;
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraph_t graph = nullptr;
  std::vector<void*> allocs;
  std::string err;
  size_t device_bytes = 0;
};

namespace {

tg_status bfail(tg_batch* b, tg_status st, const std::string& msg) {
  if (b) b->err = msg;
  g_batch_error = msg;
  return st;
}

#define TB_CUDA(b, call)                                                                          \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      return bfail((b), TG_CUDA_ERROR, std::string(#call " failed: ") + cudaGetErrorString(e_)); \
  } while (0)

template <class T>
tg_status balloc(tg_batch* b, size_t n, T** out) {
  void* p = nullptr;
  const size_t bytes = std::max<size_t>(1, n) * sizeof(T);
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) return bfail(b, TG_CUDA_ERROR, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  b->allocs.push_back(p);
  b->device_bytes += bytes;
  e = cudaMemset(p, 0, bytes);
  if (e != cudaSuccess) return bfail(b, TG_CUDA_ERROR, std::string("cudaMemset: ") + cudaGetErrorString(e));
  *out = (T*)p;
  return TG_OK;
}

template <class T, class U>
tg_status bupload(tg_batch* b, const std::vector<U>& v, const T** out) {
  T* p = nullptr;
  tg_status st = balloc(b, v.size(), &p);
  if (st != TG_OK) return st;
  std::vector<T> tmp(v.begin(), v.end());
  if (!tmp.empty()) TB_CUDA(b, cudaMemcpy(p, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice));
  *out = p;
  return TG_OK;
}

tg_status bsync(tg_batch* b) {
  TB_CUDA(b, cudaGetLastError());
  TB_CUDA(b, cudaStreamSynchronize(b->stream));
  return TG_OK;
}

// Sets the warp offsets of every level for sample tile ST over its items of
// the given kind (IT_VERTEX ...); returns the total.
template <int ST>
long long layout_warps(Batch& B, int kind) {
  long long w = 0;
  for (int l = 0; l < B.nlev; ++l) {
    B.lev[l].w_begin = w;
    w += level_warps<ST>(item_count(B.lev[l].m, kind), B.lev[l].S);
  }
  B.work = w;
  return w;
}

long long layout(Batch& B, int st, int kind) { return st == 32 ? layout_warps<32>(B, kind) : layout_warps<16>(B, kind); }

// The same for the paired kernels (H pairs of samples per lane).
template <int ST, int H>
long long layout_warps_pair(Batch& B, int kind) {
  long long w = 0;
  for (int l = 0; l < B.nlev; ++l) {
    B.lev[l].w_begin = w;
    w += level_warps_pair<ST, H>(item_count(B.lev[l].m, kind), B.lev[l].S);
  }
  B.work = w;
  return w;
}

// h pairs of samples per lane (edges and viscous units 1; the vertex kernels kLanePairs,
// the gradients of meshes with boundaries 1).
long long layout_pair(Batch& B, int st, int kind, int h) {
  if (h == 1) return st == 32 ? layout_warps_pair<32, 1>(B, kind) : layout_warps_pair<16, 1>(B, kind);
  return st == 32 ? layout_warps_pair<32, kLanePairs>(B, kind) : layout_warps_pair<16, kLanePairs>(B, kind);
}

typedef void (*FluxK)(Batch, BParams, int);

template <int F, int R>
FluxK flux_kernel_fr(int shape) {
  switch (shape) {
    case 0: return kb_edge_flux<F, R, 32, 256>;
    case 1: return kb_edge_flux<F, R, 32, 128>;
    case 2: return kb_edge_flux<F, R, 16, 256>;
    default: return kb_edge_flux<F, R, 16, 128>;
  }
}

template <int F>
FluxK flux_kernel_f(int recon, int shape) {
  return recon == RECON_FIRST ? flux_kernel_fr<F, RECON_FIRST>(shape) : flux_kernel_fr<F, RECON_TVD_MINMOD>(shape);
}

FluxK flux_kernel(int flux, int recon, int shape) {
  switch (flux) {
    case FLUX_TECNO_ROE: return flux_kernel_f<FLUX_TECNO_ROE>(recon, shape);
    case FLUX_TECNO_RUSANOV: return flux_kernel_f<FLUX_TECNO_RUSANOV>(recon, shape);
    default: return flux_kernel_fr<FLUX_KEPEC, RECON_FIRST>(shape);
  }
}

template <bool BND>
FluxK gather_kernel_b(int shape) {
  switch (shape) {
    case 0: return kb_gather_update<32, 256, BND>;
    case 1: return kb_gather_update<32, 128, BND>;
    case 2: return kb_gather_update<16, 256, BND>;
    default: return kb_gather_update<16, 128, BND>;
  }
}

FluxK gather_kernel(int shape, bool bnd) { return bnd ? gather_kernel_b<true>(shape) : gather_kernel_b<false>(shape); }

template <int F>
FluxK bflux_kernel_f(int shape) {
  switch (shape) {
    case 0: return kb_bflux<F, 32, 256>;
    case 1: return kb_bflux<F, 32, 128>;
    case 2: return kb_bflux<F, 16, 256>;
    default: return kb_bflux<F, 16, 128>;
  }
}

FluxK bflux_kernel(int flux, int shape) {
  switch (flux) {
    case FLUX_TECNO_ROE: return bflux_kernel_f<FLUX_TECNO_ROE>(shape);
    case FLUX_TECNO_RUSANOV: return bflux_kernel_f<FLUX_TECNO_RUSANOV>(shape);
    default: return bflux_kernel_f<FLUX_KEPEC>(shape);
  }
}

FluxK viscous_kernel(int shape) {
  switch (shape) {
    case 0: return kb_viscous<32, 256>;
    case 1: return kb_viscous<32, 128>;
    case 2: return kb_viscous<16, 256>;
    default: return kb_viscous<16, 128>;
  }
}

typedef void (*GradK)(Batch, BParams, int, int);

GradK grad_kernel(int st, bool bnd) {
  if (st == 32) return bnd ? kb_grad<32, true> : kb_grad<32, false>;
  return bnd ? kb_grad<16, true> : kb_grad<16, false>;
}

bool needs_grad(const tg_batch* b) {
  return b->prm.recon != RECON_FIRST && (b->prm.flux == FLUX_TECNO_ROE || b->prm.flux == FLUX_TECNO_RUSANOV);
}

int max_samples(const tg_batch* b) {
  int m = 0;
  for (int l = 0; l < b->nlev; ++l) m = std::max(m, b->B.lev[l].S);
  return m;
}

unsigned blocks_of(const Batch& B, int bs) { return (unsigned)((B.work * 32 + bs - 1) / bs); }

// One full step of every level on b->stream.
void enqueue_step(tg_batch* b) {
  const Shape sh = kShapes[b->shape];
  Batch B = b->B, BG = b->B, BE = b->B, BB = b->B, BU = b->B;
  layout_pair(B, sh.st, IT_VERTEX, kLanePairs);
  layout_pair(BG, sh.st, IT_VERTEX, b->bnd ? 1 : kLanePairs);   // as kb_grad's default
  layout_pair(BE, sh.st, IT_EDGE, 1);
  layout(BB, sh.st, IT_BSLOT);
  layout_pair(BU, sh.st, IT_UNIT, 1);
  const dim3 gs((max_samples(b) + 255) / 256, b->nlev);
  kb_step_begin<<<gs, 256, 0, b->stream>>>(B, b->prm);
  long long dt_blocks = 0;
  for (int l = 0; l < b->nlev; ++l) dt_blocks += (long long)dt_groups(B.lev[l].S) * b->dt_chunks;
  if (b->bnd) kb_dt<8, true><<<(unsigned)dt_blocks, 256, 0, b->stream>>>(B, b->prm, b->dt_chunks);
  else kb_dt<8, false><<<(unsigned)dt_blocks, 256, 0, b->stream>>>(B, b->prm, b->dt_chunks);
  kb_dt_final<<<gs, 256, 0, b->stream>>>(B, b->prm);
  FluxK fk = flux_kernel(b->prm.flux, b->prm.recon, b->shape);
  FluxK gk = gather_kernel(b->shape, b->bnd);
  GradK rk = grad_kernel(sh.st, b->bnd);
  for (int r = 0; r < 3; ++r) {
    if (needs_grad(b)) rk<<<blocks_of(BG, sh.bs), sh.bs, 0, b->stream>>>(BG, b->prm, r, 0);
    if (b->bnd && BB.work > 0) bflux_kernel(b->prm.flux, b->shape)<<<blocks_of(BB, sh.bs), sh.bs, 0, b->stream>>>(BB, b->prm, r);
    if (b->prm.model == 1) viscous_kernel(b->shape)<<<blocks_of(BU, sh.bs), sh.bs, 0, b->stream>>>(BU, b->prm, r);
    fk<<<blocks_of(BE, sh.bs), sh.bs, 0, b->stream>>>(BE, b->prm, r);
    gk<<<blocks_of(B, sh.bs), sh.bs, 0, b->stream>>>(B, b->prm, r);
  }
  kb_step_end<<<gs, 256, 0, b->stream>>>(B, b->prm);
}

bool has_bfaces(const tg_batch* b) {
  for (int l = 0; l < b->nlev; ++l)
    if (b->B.lev[l].m.nb > 0) return true;
  return false;
}

int kernels_per_step(const tg_batch* b) {
  const int per_stage = 2 + (needs_grad(b) ? 1 : 0) + (b->bnd && has_bfaces(b) ? 1 : 0) + (b->prm.model == 1 ? 1 : 0);
  return 4 + 3 * per_stage;
}

void drop_graph(tg_batch* b) {
  if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->graph_exec = nullptr;
  b->graph = nullptr;
}

tg_status capture(tg_batch* b) {
  if (b->graph_exec) return TG_OK;
  TB_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  enqueue_step(b);
  cudaError_t e = cudaStreamEndCapture(b->stream, &b->graph);
  if (e != cudaSuccess) return bfail(b, TG_CUDA_ERROR, std::string("graph capture: ") + cudaGetErrorString(e));
  TB_CUDA(b, cudaGraphInstantiate(&b->graph_exec, b->graph, 0));
  return TG_OK;
}

struct ClockHost {
  std::vector<double> elapsed;
  std::vector<int> counter, bad;
};

tg_status read_clock(tg_batch* b, int l, ClockHost& c) {
  const int S = b->B.lev[l].S;
  c.elapsed.resize(S); c.counter.resize(S); c.bad.resize(S);
  TB_CUDA(b, cudaMemcpyAsync(c.elapsed.data(), b->B.lev[l].c.elapsed, S * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
  TB_CUDA(b, cudaMemcpyAsync(c.counter.data(), b->B.lev[l].c.counter, S * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  TB_CUDA(b, cudaMemcpyAsync(c.bad.data(), b->B.lev[l].c.bad, S * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  return bsync(b);
}

// Every sample of every level is past output `instance`, finished, or bad.
tg_status all_reached(tg_batch* b, int instance, bool* yes, int* nbad) {
  *yes = true;
  *nbad = 0;
  for (int l = 0; l < b->nlev; ++l) {
    ClockHost c;
    tg_status st = read_clock(b, l, c);
    if (st != TG_OK) return st;
    for (int s = 0; s < b->B.lev[l].S; ++s) {
      if (c.bad[s]) { ++*nbad; continue; }
      if (c.counter[s] <= instance && c.elapsed[s] < b->prm.final_time) *yes = false;
    }
  }
  return TG_OK;
}

tg_status reset_clock(tg_batch* b, int l, int s0, int n) {
  const LevelClock& c = b->B.lev[l].c;
  std::vector<double> z(n, 0.0);
  std::vector<int> one(n, 1), zero(n, 0);
  TB_CUDA(b, cudaMemcpyAsync(c.elapsed + s0, z.data(), n * sizeof(double), cudaMemcpyHostToDevice, b->stream));
  TB_CUDA(b, cudaMemcpyAsync(c.counter + s0, one.data(), n * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  TB_CUDA(b, cudaMemcpyAsync(c.reached + s0, zero.data(), n * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  TB_CUDA(b, cudaMemcpyAsync(c.bad + s0, zero.data(), n * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  return bsync(b);
}

}  // namespace

extern "C" {

tg_status tg_batch_create(const tg_batch_level* levels, int n_levels, const tg_material* mat, const tg_options* opt,
                          tg_batch** out) {
  if (!out) return bfail(nullptr, TG_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (!levels || !mat || !opt || n_levels < 1 || n_levels > kMaxLevels)
    return bfail(nullptr, TG_INVALID_ARG, "need 1 to 4 levels, a material and options");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return bfail(nullptr, TG_NO_DEVICE, "no CUDA device visible; the GPU path has no CPU fallback");
  if (mat->model != 0 && mat->mu_model != 0)
    return bfail(nullptr, TG_NOT_SUPPORTED, "batched Navier-Stokes ensembles use the constant viscosity law");
  if (opt->bc_strong || opt->liou_fix)
    return bfail(nullptr, TG_NOT_SUPPORTED, "batched ensembles run weak boundary conditions without the Liou switch");
  if (!(mat->flux_scheme == FLUX_TECNO_ROE || mat->flux_scheme == FLUX_TECNO_RUSANOV || mat->flux_scheme == FLUX_KEPEC))
    return bfail(nullptr, TG_NOT_SUPPORTED, "batched ensembles run kepes_tecno_roe, kepes_tecno_rusanov or kepec");
  if (!(mat->reconstruct_scheme == RECON_FIRST || mat->reconstruct_scheme == RECON_TVD_MINMOD))
    return bfail(nullptr, TG_NOT_SUPPORTED, "batched ensembles reconstruct first order or with minmod");
  if (opt->time_scheme != TG_TIME_SSPRK3 || opt->time_mode != TG_UNSTEADY || !(opt->cfl > 0.0) || opt->time_step > 0.0 ||
      opt->n_time_stamps <= 0)
    return bfail(nullptr, TG_NOT_SUPPORTED, "batched ensembles run unsteady SSP-RK3 with a CFL time step");
  tg_batch* b = new (std::nothrow) tg_batch();
  if (!b) return bfail(nullptr, TG_INVALID_ARG, "out of host memory");
  cudaGetDevice(&b->device);
  b->nlev = n_levels;
  b->B.nlev = n_levels;
  tg_status st;
  for (int l = 0; l < n_levels; ++l) {
    if (!levels[l].mesh || levels[l].n_samples < 32 || levels[l].n_samples % 32 != 0) {
      tg_batch_destroy(b);
      return bfail(nullptr, TG_INVALID_ARG, "every level needs a mesh and a positive multiple of 32 samples");
    }
    if (levels[l].mesh->vertex_radius) {
      tg_batch_destroy(b);
      return bfail(nullptr, TG_NOT_SUPPORTED, "batched ensembles run planar meshes (no radii)");
    }
    LevelHost& H = b->lh[l];
    std::string msg = build_layout(*levels[l].mesh, levels[l].bc, mat->model == 1, H.L);
    if (!msg.empty()) { tg_batch_destroy(b); return bfail(nullptr, TG_INVALID_ARG, msg); }
    if (H.L.nb != 0 || mat->model == 1) b->bnd = true;
    H.S = levels[l].n_samples;
    const HostLayout& L = H.L;
    Level& V = b->B.lev[l];
    V.S = H.S;
    V.P = H.S + 32;
    LevelMesh& m = V.m;
    m.nv = L.nv; m.ne = L.ne;
    // geometry formed in FP64, stored in FP32
    std::vector<double> ux(L.ne), uy(L.ne), ar(L.ne), aw(L.nv), visw(L.nv, 0.0);
    for (int v = 0; v < L.nv; ++v) aw[v] = L.dcarea[v] * L.pweight[v];
    for (int v = 0; v < L.nv; ++v)
      for (int j = L.ce_off[v]; j < L.ce_off[v + 1]; ++j) {
        const int e = L.ce_ent[j] >> 1;
        visw[v] += std::sqrt(L.e_nx[e] * L.e_nx[e] + L.e_ny[e] * L.e_ny[e]) /
                   std::sqrt(L.e_dx[e] * L.e_dx[e] + L.e_dy[e] * L.e_dy[e]);
      }
    for (int e = 0; e < L.ne; ++e) {
      const double a = std::sqrt(L.e_nx[e] * L.e_nx[e] + L.e_ny[e] * L.e_ny[e]);
      const double ia = a > 0.0 ? 1.0 / a : 0.0;   // gradient-only edges carry no flux
      ux[e] = L.e_nx[e] * ia; uy[e] = L.e_ny[e] * ia; ar[e] = a;
    }
#define BU(vec, field) \
    if ((st = bupload(b, vec, &m.field)) != TG_OK) { tg_batch_destroy(b); return st; }
    BU(L.e_a, e_a) BU(L.e_b, e_b) BU(ux, ux) BU(uy, uy) BU(ar, ar) BU(L.e_nx, nx) BU(L.e_ny, ny)
    BU(L.e_dx, dx) BU(L.e_dy, dy) BU(L.e_g0x, g0x) BU(L.e_g0y, g0y) BU(L.e_g1x, g1x) BU(L.e_g1y, g1y)
    BU(L.ce_off, ce_off) BU(L.ce_ent, ce_ent) BU(L.dcarea, area) BU(L.inv6mc, inv6mc) BU(visw, visw) BU(L.x, x) BU(L.y, y) BU(aw, aw)
    m.nb = L.nb; m.nvu = L.nvu; m.nic = L.n_int_cells;
    BU(L.b_v0, b_v0) BU(L.b_v1, b_v1) BU(L.b_kind, b_kind) BU(L.b_adiab, b_adiab) BU(L.b_nx, b_nx) BU(L.b_ny, b_ny)
    BU(L.cb_off, cb_off) BU(L.cb_ent, cb_ent)
    BU(L.u_cell, u_cell) BU(L.c_v, c_v) BU(L.c_n, c_n) BU(L.c_inv2a, c_inv2a) BU(L.c_bf_off, c_bf_off) BU(L.c_bf, c_bf)
    BU(L.c_nbr_off, c_nbr_off) BU(L.c_nbr, c_nbr) BU(L.bf_face_nx, bf_nx) BU(L.bf_face_ny, bf_ny)
    BU(L.bf_face_v0, bf_v0) BU(L.bf_face_v1, bf_v1)
#undef BU
    const size_t vs = (size_t)L.nv * V.P;
    for (int r = 0; r < 3; ++r)
      if ((st = balloc(b, kQ * vs, &V.Q[r])) != TG_OK) { tg_batch_destroy(b); return st; }
    if ((st = balloc(b, 4 * vs, &V.Uold)) != TG_OK) { tg_batch_destroy(b); return st; }
    if ((st = balloc(b, 4 * (size_t)L.ne * V.P, &V.F)) != TG_OK) { tg_batch_destroy(b); return st; }
    if ((mat->reconstruct_scheme != RECON_FIRST && mat->flux_scheme != FLUX_KEPEC) || L.nb > 0 || mat->model == 1) {
      if ((st = balloc(b, kG * vs, &V.G)) != TG_OK) { tg_batch_destroy(b); return st; }
    }
    if (L.nb > 0 || mat->model == 1) {
      // per-sample boundary values and viscosity, initialised from the level's table and the material
      if ((st = balloc(b, 10 * (size_t)std::max(L.nb, 1) * V.P, &V.bval)) != TG_OK ||
          (st = balloc(b, (size_t)V.P, &V.mu)) != TG_OK ||
          (st = balloc(b, 8 * (size_t)std::max(L.nb, 1) * V.P, &V.Fb)) != TG_OK ||
          (st = balloc(b, 3 * (size_t)std::max(L.nb, 1) * V.P, &V.Fvb)) != TG_OK ||
          (st = balloc(b, 9 * (size_t)std::max(L.nvu, 1) * V.P, &V.Fv)) != TG_OK) {
        tg_batch_destroy(b);
        return st;
      }
    }
    LevelClock& c = V.c;
    if ((st = balloc(b, H.S, &c.elapsed)) != TG_OK || (st = balloc(b, H.S, &c.dt)) != TG_OK ||
        (st = balloc(b, H.S, &c.dtmin_bits)) != TG_OK || (st = balloc(b, H.S, &c.counter)) != TG_OK ||
        (st = balloc(b, H.S, &c.reached)) != TG_OK || (st = balloc(b, H.S, &c.active)) != TG_OK ||
        (st = balloc(b, H.S, &c.bad)) != TG_OK) {
      tg_batch_destroy(b);
      return st;
    }
  }
  // the kernels index a launch's warps in 32 bits
  for (int kind : {IT_VERTEX, IT_EDGE, IT_BSLOT, IT_UNIT}) {
    Batch tmp = b->B;
    if (layout_warps<16>(tmp, kind) >= (1LL << 31) || layout_warps<32>(tmp, kind) >= (1LL << 31)) {
      tg_batch_destroy(b);
      return bfail(nullptr, TG_INVALID_ARG, "batch too large: a launch exceeds 2^31 warps");
    }
  }
  BParams& k = b->prm;
  k.gamma = (float)mat->gamma; k.R = (float)mat->gas_const;
  k.inv_gm1 = (float)(1.0 / (mat->gamma - 1.0)); k.inv_gamma = (float)(1.0 / mat->gamma);
  k.sqrt_gm1 = (float)std::sqrt(mat->gamma - 1.0); k.cfl = (float)opt->cfl;
  k.ev_alpha = (float)mat->ev_mod_alpha; k.ev_beta = (float)mat->ev_mod_beta;
  k.final_time = opt->final_time;
  k.flux = mat->flux_scheme; k.recon = mat->reconstruct_scheme;
  k.model = mat->model;
  k.cp_over_pr = (float)(mat->gamma * mat->gas_const / (mat->gamma - 1.0) / mat->prandtl);
  k.visc = mat->visc_active; k.heat = mat->heat_active;
  // output time instances (src/fv.cc:52-62)
  std::vector<double> ti;
  const double dti = opt->final_time / opt->n_time_stamps;
  for (int i = 0; i <= opt->n_time_stamps; ++i) ti.push_back(i * dti);
  const double* tip = nullptr;
  if ((st = bupload(b, ti, &tip)) != TG_OK) { tg_batch_destroy(b); return st; }
  k.tinst = tip;
  k.ntinst = (int)ti.size();
  if ((st = balloc(b, 1, &b->stop)) != TG_OK) { tg_batch_destroy(b); return st; }
  k.stop_counter = INT_MAX;
  k.stop = b->stop;
  int inf = INT_MAX;
  cudaMemcpy(b->stop, &inf, sizeof(int), cudaMemcpyHostToDevice);
  // dt kernel: about four blocks per SM over all sample groups
  long long groups = 0;
  for (int l = 0; l < n_levels; ++l) groups += dt_groups(b->B.lev[l].S);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  b->dt_chunks = (int)std::max<long long>(1, (4LL * sms + groups - 1) / groups);
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { tg_batch_destroy(b); return bfail(nullptr, TG_CUDA_ERROR, cudaGetErrorString(e)); }
  for (int l = 0; l < n_levels; ++l)
    if ((st = reset_clock(b, l, 0, b->B.lev[l].S)) != TG_OK) { tg_batch_destroy(b); return st; }
  for (int l = 0; l < n_levels; ++l) {
    if (!b->B.lev[l].mu) continue;
    const int S = b->B.lev[l].S;
    const size_t nbf = b->lh[l].L.rb_type.size();
    std::vector<double> mu(S, mat->mu_ref), bv;
    const double* bvp = nullptr;
    if (levels[l].bc && levels[l].bc->bface_values && nbf) {
      bv.resize((size_t)S * nbf * 10);
      for (int s = 0; s < S; ++s) std::memcpy(bv.data() + (size_t)s * nbf * 10, levels[l].bc->bface_values, nbf * 10 * sizeof(double));
      bvp = bv.data();
    }
    if ((st = tg_batch_set_parameters(b, l, mu.data(), bvp)) != TG_OK) { tg_batch_destroy(b); return st; }
  }
  *out = b;
  return TG_OK;
}

tg_status tg_batch_destroy(tg_batch* b) {
  if (!b) return TG_OK;
  drop_graph(b);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (void* p : b->allocs) cudaFree(p);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return TG_OK;
}

const char* tg_batch_last_error(const tg_batch* b) { return b ? b->err.c_str() : g_batch_error.c_str(); }

tg_status tg_batch_set_state(tg_batch* b, int level, int sample, const double* prim_aos, int n_vertex) {
  if (!b || !prim_aos || level < 0 || level >= b->nlev) return bfail(b, TG_INVALID_ARG, "bad level or NULL state");
  const Level& V = b->B.lev[level];
  const HostLayout& L = b->lh[level].L;
  if (sample < 0 || sample >= V.S || n_vertex != L.nv) return bfail(b, TG_INVALID_ARG, "bad sample or vertex count");
  std::vector<float> q((size_t)kQ * L.nv);
  const double g = b->prm.gamma;
  for (int i = 0; i < L.nv; ++i) {
    const double* p = prim_aos + 5 * (size_t)L.old_of_new[i];   // PrimVar T, p, u, v, w
    const double T = p[0], pr = p[1], u = p[2], v = p[3];
    if (!(T > 0.0) || !(pr > 0.0)) return bfail(b, TG_INVALID_ARG, "state needs T > 0 and p > 0 (src/fv.cc:388-389)");
    const double rho = pr / (b->prm.R * T);
    const double beta = rho / (2.0 * pr);
    const double s = std::log(pr) - g * std::log(rho);
    float* r = q.data() + (size_t)kQ * i;     // device rows [vertex][component]
    r[0] = (float)u;
    r[1] = (float)v;
    r[2] = (float)pr;
    r[3] = (float)((g - s) / (g - 1.0) - (u * u + v * v) * beta);
    r[4] = (float)(-2.0 * beta);
  }
  TB_CUDA(b, cudaMemcpy2DAsync(V.Q[0] + sample, V.P * sizeof(float), q.data(), sizeof(float), sizeof(float),
                               (size_t)kQ * L.nv, cudaMemcpyHostToDevice, b->stream));
  return reset_clock(b, level, sample, 1);
}

tg_status tg_batch_get_state(tg_batch* b, int level, int sample, double* prim_aos, int n_vertex) {
  if (!b || !prim_aos || level < 0 || level >= b->nlev) return bfail(b, TG_INVALID_ARG, "bad level or NULL state");
  const Level& V = b->B.lev[level];
  const HostLayout& L = b->lh[level].L;
  if (sample < 0 || sample >= V.S || n_vertex != L.nv) return bfail(b, TG_INVALID_ARG, "bad sample or vertex count");
  std::vector<float> q((size_t)kQ * L.nv);
  TB_CUDA(b, cudaMemcpy2DAsync(q.data(), sizeof(float), V.Q[0] + sample, V.P * sizeof(float), sizeof(float),
                               (size_t)kQ * L.nv, cudaMemcpyDeviceToHost, b->stream));
  tg_status st = bsync(b);
  if (st != TG_OK) return st;
  for (int i = 0; i < L.nv; ++i) {
    double* p = prim_aos + 5 * (size_t)L.old_of_new[i];
    const float* r = q.data() + (size_t)kQ * i;
    const double u = r[0], v = r[1], pr = r[2], V5 = r[4];
    const double rho = -V5 * pr;
    p[0] = pr / (b->prm.R * rho); p[1] = pr; p[2] = u; p[3] = v; p[4] = 0.0;
  }
  return TG_OK;
}

tg_status tg_batch_set_parameters(tg_batch* b, int level, const double* mu_ref, const double* bface_values) {
  if (!b || level < 0 || level >= b->nlev) return bfail(b, TG_INVALID_ARG, "bad level");
  const Level& V = b->B.lev[level];
  const HostLayout& L = b->lh[level].L;
  if (!V.mu) return bfail(b, TG_NOT_SUPPORTED, "a periodic Euler level has no per-sample parameters");
  const int S = V.S;
  if (mu_ref) {
    std::vector<float> mu(V.P, 0.0f);
    for (int s = 0; s < S; ++s) {
      if (!(mu_ref[s] >= 0.0)) return bfail(b, TG_INVALID_ARG, "viscosity must be >= 0");
      mu[s] = (float)mu_ref[s];
    }
    TB_CUDA(b, cudaMemcpyAsync(V.mu, mu.data(), V.P * sizeof(float), cudaMemcpyHostToDevice, b->stream));
  }
  if (bface_values && L.nb > 0) {
    // reference boundary-face order (10 values per face) -> [device face][value][sample]
    const size_t nbf = L.rb_type.size();
    std::vector<float> h((size_t)L.nb * 10 * V.P, 0.0f);
    for (size_t f = 0; f < nbf; ++f) {
      const int d = L.rb_dev[f];
      if (d < 0) continue;
      for (int q = 0; q < 10; ++q) {
        float* row = h.data() + ((size_t)d * 10 + q) * V.P;
        for (int s = 0; s < S; ++s) row[s] = (float)bface_values[((size_t)s * nbf + f) * 10 + q];
      }
    }
    TB_CUDA(b, cudaMemcpyAsync(V.bval, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, b->stream));
  }
  return bsync(b);
}

tg_status tg_batch_set_uniform(tg_batch* b, int level, const double* prim) {
  if (!b || !prim || level < 0 || level >= b->nlev) return bfail(b, TG_INVALID_ARG, "bad level or NULL state");
  const Level& V = b->B.lev[level];
  const int S = V.S;
  const double g = b->prm.gamma;
  std::vector<float> rec((size_t)kQ * S);
  for (int s = 0; s < S; ++s) {
    const double* p = prim + 5 * (size_t)s;   // PrimVar T, p, u, v, w
    const double T = p[0], pr = p[1], u = p[2], v = p[3];
    if (!(T > 0.0) || !(pr > 0.0)) return bfail(b, TG_INVALID_ARG, "state needs T > 0 and p > 0 (src/fv.cc:388-389)");
    const double rho = pr / (b->prm.R * T);
    const double beta = rho / (2.0 * pr);
    const double ent = std::log(pr) - g * std::log(rho);
    rec[0 * (size_t)S + s] = (float)u;
    rec[1 * (size_t)S + s] = (float)v;
    rec[2 * (size_t)S + s] = (float)pr;
    rec[3 * (size_t)S + s] = (float)((g - ent) / (g - 1.0) - (u * u + v * v) * beta);
    rec[4 * (size_t)S + s] = (float)(-2.0 * beta);
  }
  float* d = nullptr;
  TB_CUDA(b, cudaMalloc((void**)&d, rec.size() * sizeof(float)));
  cudaError_t e = cudaMemcpyAsync(d, rec.data(), rec.size() * sizeof(float), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) {
    const long long t = (long long)V.m.nv * S;
    kb_ic_uniform<<<(unsigned)((t + 255) / 256), 256, 0, b->stream>>>(V, d);
    e = cudaStreamSynchronize(b->stream);
  }
  cudaFree(d);
  if (e != cudaSuccess) return bfail(b, TG_CUDA_ERROR, cudaGetErrorString(e));
  return reset_clock(b, level, 0, S);
}

tg_status tg_batch_forces(tg_batch* b, int level, int n_forces, const int* n_tags, const int* tags, double* out) {
  if (!b || level < 0 || level >= b->nlev || n_forces < 1 || !n_tags || !tags || !out)
    return bfail(b, TG_INVALID_ARG, "bad level or force specification");
  const Level& V = b->B.lev[level];
  if (!V.mu) return bfail(b, TG_NOT_SUPPORTED, "a periodic Euler level has no boundary faces");
  std::vector<int> rec4, off;
  const std::string msg = force_faces(b->lh[level].L, n_forces, n_tags, tags, rec4, off);
  if (!msg.empty()) return bfail(b, TG_INVALID_ARG, msg);
  // the viscous force reads the vertex gradients of the current state (src/force.cc:123)
  const Shape sh = kShapes[0];
  Batch B = b->B;
  layout_pair(B, sh.st, IT_VERTEX, 1);   // kb_grad<*, true> takes one pair per lane
  if (b->prm.model == 1) grad_kernel(sh.st, true)<<<blocks_of(B, sh.bs), sh.bs, 0, b->stream>>>(B, b->prm, 0, 1);
  int* drec = nullptr;
  int* doff = nullptr;
  double* dout = nullptr;
  const size_t nout = (size_t)V.S * n_forces * 4;
  TB_CUDA(b, cudaMalloc((void**)&drec, rec4.size() * sizeof(int)));
  cudaError_t e = cudaMalloc((void**)&doff, off.size() * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void**)&dout, nout * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyAsync(drec, rec4.data(), rec4.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(doff, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) {
    kb_forces<8><<<(unsigned)(n_forces * (V.S >> 5)), 256, 0, b->stream>>>(V, b->prm, (const int4*)drec, doff, n_forces, dout);
    e = cudaMemcpyAsync(out, dout, nout * sizeof(double), cudaMemcpyDeviceToHost, b->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaFree(drec);
  cudaFree(doff);
  cudaFree(dout);
  if (e != cudaSuccess) return bfail(b, TG_CUDA_ERROR, cudaGetErrorString(e));
  return TG_OK;
}

namespace {

// Device copies of five packed programs and the samples' random numbers.
struct ExprUpload {
  int *code = nullptr, *off = nullptr, *err = nullptr;
  double *k = nullptr, *rnd = nullptr;
  ~ExprUpload() { cudaFree(code); cudaFree(off); cudaFree(err); cudaFree(k); cudaFree(rnd); }
  cudaError_t load(const tg_expr* const* fields, const double* rnd_rows, size_t n_rnd_total, cudaStream_t st) {
    std::vector<int> c, o;
    std::vector<double> kk;
    expr::pack5(fields, nullptr, c, o, kk);
    cudaError_t e = cudaMalloc((void**)&code, c.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void**)&off, o.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void**)&k, std::max<size_t>(1, kk.size()) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void**)&rnd, std::max<size_t>(1, n_rnd_total) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void**)&err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpyAsync(code, c.data(), c.size() * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(off, o.data(), o.size() * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !kk.empty()) e = cudaMemcpyAsync(k, kk.data(), kk.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && n_rnd_total) e = cudaMemcpyAsync(rnd, rnd_rows, n_rnd_total * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), st);
    return e;
  }
  expr::Field5 view() const { return expr::Field5{code, off, k}; }
};

}  // namespace

tg_status tg_batch_set_state_expr(tg_batch* b, int level, const tg_expr* const* fields, const double* rnd_rows,
                                  int n_rnd) {
  if (!b || !fields || level < 0 || level >= b->nlev) return bfail(b, TG_INVALID_ARG, "bad level or NULL fields");
  for (int c = 0; c < 5; ++c)
    if (c != 3 && !fields[c]) return bfail(b, TG_INVALID_ARG, "temperature, velocity and pressure expressions are needed");
  const Level& V = b->B.lev[level];
  if (n_rnd < 0 || (n_rnd > 0 && !rnd_rows)) return bfail(b, TG_INVALID_ARG, "bad random numbers");
  ExprUpload up;
  cudaError_t e = up.load(fields, rnd_rows, (size_t)V.S * n_rnd, b->stream);
  int err = 0;
  if (e == cudaSuccess) {
    const long long t = (long long)V.m.nv * V.S;
    kb_ic_expr<<<(unsigned)((t + 255) / 256), 256, 0, b->stream>>>(V, b->prm, up.view(), up.rnd, n_rnd, up.err);
    e = cudaMemcpyAsync(&err, up.err, sizeof(int), cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  }
  if (e != cudaSuccess) return bfail(b, TG_CUDA_ERROR, cudaGetErrorString(e));
  if (err & 8) return bfail(b, TG_INVALID_ARG, "an initial state has T <= 0 or p <= 0 (src/fv.cc:388-389)");
  if (err) return bfail(b, TG_INVALID_ARG, "pert: unknown type or random-number index out of range");
  return reset_clock(b, level, 0, V.S);
}

tg_status tg_batch_set_bc_expr(tg_batch* b, int level, int tag, const tg_expr* const* fields, const double* rnd_rows,
                               int n_rnd, double t) {
  if (!b || !fields || level < 0 || level >= b->nlev) return bfail(b, TG_INVALID_ARG, "bad level or NULL fields");
  const Level& V = b->B.lev[level];
  const HostLayout& L = b->lh[level].L;
  if (!V.bval) return bfail(b, TG_NOT_SUPPORTED, "a periodic Euler level has no boundary values");
  if (n_rnd < 0 || (n_rnd > 0 && !rnd_rows)) return bfail(b, TG_INVALID_ARG, "bad random numbers");
  int mask = 0;
  for (int c = 0; c < 5; ++c) mask |= fields[c] ? (1 << c) : 0;
  std::vector<int> btag(std::max(L.nb, 1), INT_MIN);
  bool any = false;
  for (size_t f = 0; f < L.rb_type.size(); ++f)
    if (L.rb_dev[f] >= 0) { btag[L.rb_dev[f]] = L.rb_type[f]; any = any || L.rb_type[f] == tag; }
  if (!any) return bfail(b, TG_INVALID_ARG, "no non-periodic boundary face has this tag");
  ExprUpload up;
  int* dtag = nullptr;
  cudaError_t e = up.load(fields, rnd_rows, (size_t)V.S * n_rnd, b->stream);
  if (e == cudaSuccess) e = cudaMalloc((void**)&dtag, btag.size() * sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyAsync(dtag, btag.data(), btag.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream);
  int err = 0;
  if (e == cudaSuccess) {
    const long long n = 2LL * L.nb * V.S;
    kb_bc_expr<<<(unsigned)((n + 255) / 256), 256, 0, b->stream>>>(V, up.view(), mask, dtag, tag, up.rnd, n_rnd, t,
                                                                   up.err);
    e = cudaMemcpyAsync(&err, up.err, sizeof(int), cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  }
  cudaFree(dtag);
  if (e != cudaSuccess) return bfail(b, TG_CUDA_ERROR, cudaGetErrorString(e));
  if (err) return bfail(b, TG_INVALID_ARG, "pert: unknown type or random-number index out of range");
  return TG_OK;
}

tg_status tg_batch_set_kh(tg_batch* b, int level, const double* rows, int n_rnd) {
  if (!b || !rows || level < 0 || level >= b->nlev || n_rnd < 2 || n_rnd % 2)
    return bfail(b, TG_INVALID_ARG, "bad level, NULL rows or odd row length");
  const Level& V = b->B.lev[level];
  double* d = nullptr;
  const size_t n = (size_t)V.S * n_rnd;
  TB_CUDA(b, cudaMalloc((void**)&d, n * sizeof(double)));
  cudaError_t e = cudaMemcpyAsync(d, rows, n * sizeof(double), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) {
    const long long t = (long long)V.m.nv * V.S;
    kb_ic_kh<<<(unsigned)((t + 255) / 256), 256, 0, b->stream>>>(V, b->prm, d, n_rnd);
    e = cudaStreamSynchronize(b->stream);
  }
  cudaFree(d);
  if (e != cudaSuccess) return bfail(b, TG_CUDA_ERROR, cudaGetErrorString(e));
  return reset_clock(b, level, 0, V.S);
}

tg_status tg_batch_advance(tg_batch* b, int instance, long max_steps, double* info4) {
  if (!b) return bfail(b, TG_INVALID_ARG, "NULL batch");
  if (max_steps < 0) return bfail(b, TG_INVALID_ARG, "max_steps < 0");
  tg_status st = capture(b);
  if (st != TG_OK) return st;
  TB_CUDA(b, cudaMemcpyAsync(b->stop, &instance, sizeof(int), cudaMemcpyHostToDevice, b->stream));
  bool done = false;
  int nbad = 0;
  long launched = 0;
  if ((st = all_reached(b, instance, &done, &nbad)) != TG_OK) return st;
  while (!done && launched < max_steps) {
    const long chunk = std::min<long>(8, max_steps - launched);
    for (long i = 0; i < chunk; ++i) TB_CUDA(b, cudaGraphLaunch(b->graph_exec, b->stream));
    launched += chunk;
    if ((st = all_reached(b, instance, &done, &nbad)) != TG_OK) return st;
  }
  int inf = INT_MAX;
  TB_CUDA(b, cudaMemcpyAsync(b->stop, &inf, sizeof(int), cudaMemcpyHostToDevice, b->stream));
  if ((st = bsync(b)) != TG_OK) return st;
  if (info4) {
    double lo = 1e300, hi = -1e300;
    for (int l = 0; l < b->nlev; ++l) {
      ClockHost c;
      if ((st = read_clock(b, l, c)) != TG_OK) return st;
      for (double x : c.elapsed) { lo = std::min(lo, x); hi = std::max(hi, x); }
    }
    info4[0] = (double)launched; info4[1] = lo; info4[2] = hi; info4[3] = (double)nbad;
  }
  if (nbad) return bfail(b, TG_BAD_STATE, std::to_string(nbad) + " sample(s) produced a non-finite or non-positive state");
  return TG_OK;
}

tg_status tg_batch_clock(tg_batch* b, int level, double* elapsed, int* counter, int* bad) {
  if (!b || level < 0 || level >= b->nlev) return bfail(b, TG_INVALID_ARG, "bad level");
  ClockHost c;
  tg_status st = read_clock(b, level, c);
  if (st != TG_OK) return st;
  const int S = b->B.lev[level].S;
  if (elapsed) std::memcpy(elapsed, c.elapsed.data(), S * sizeof(double));
  if (counter) std::memcpy(counter, c.counter.data(), S * sizeof(int));
  if (bad) std::memcpy(bad, c.bad.data(), S * sizeof(int));
  return TG_OK;
}

tg_status tg_batch_moments(tg_batch* b, int level, int extras, double* fm, double* sm, double* m2) {
  if (!b || level < 0 || level >= b->nlev || extras < 0 || extras > 7)
    return bfail(b, TG_INVALID_ARG, "bad level or extras (density, mach, entropy: bits 1, 2, 4)");
  const Level& V = b->B.lev[level];
  const HostLayout& L = b->lh[level].L;
  const int nvar = 5 + (extras & 1) + ((extras >> 1) & 1) + ((extras >> 2) & 1);
  const size_t n = (size_t)nvar * L.nv;
  double* d = nullptr;
  TB_CUDA(b, cudaMalloc((void**)&d, 3 * n * sizeof(double)));
  kb_moments<<<(unsigned)((n + 127) / 128), 128, 0, b->stream>>>(V, b->prm, extras, nvar, d, d + n, d + 2 * n);
  std::vector<double> h(3 * n);
  cudaError_t e = cudaMemcpyAsync(h.data(), d, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  cudaFree(d);
  if (e != cudaSuccess) return bfail(b, TG_CUDA_ERROR, cudaGetErrorString(e));
  double* out[3] = {fm, sm, m2};
  for (int w = 0; w < 3; ++w) {
    if (!out[w]) continue;
    for (int i = 0; i < L.nv; ++i) {
      double* dst = out[w] + (size_t)nvar * L.old_of_new[i];
      for (int c = 0; c < nvar; ++c) dst[c] = h[(size_t)w * n + (size_t)c * L.nv + i];
    }
  }
  return TG_OK;
}

tg_status tg_batch_integrals(tg_batch* b, int level, double* out) {
  if (!b || !out || level < 0 || level >= b->nlev) return bfail(b, TG_INVALID_ARG, "bad level or NULL output");
  const Level& V = b->B.lev[level];
  const int chunks = 16;
  double* d = nullptr;
  const size_t n = (size_t)chunks * V.S * 3;
  TB_CUDA(b, cudaMalloc((void**)&d, n * sizeof(double)));
  kb_integrals<8><<<(V.S >> 5) * chunks, 256, 0, b->stream>>>(V, b->prm, chunks, d);
  std::vector<double> h(n);
  cudaError_t e = cudaMemcpyAsync(h.data(), d, n * sizeof(double), cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  cudaFree(d);
  if (e != cudaSuccess) return bfail(b, TG_CUDA_ERROR, cudaGetErrorString(e));
  for (int s = 0; s < V.S; ++s)
    for (int c = 0; c < 3; ++c) {
      double acc = 0.0;
      for (int ch = 0; ch < chunks; ++ch) acc += h[((size_t)ch * V.S + s) * 3 + c];
      out[(size_t)s * 3 + c] = acc;
    }
  return TG_OK;
}

tg_status tg_batch_set_shape(tg_batch* b, int shape) {
  if (!b || shape < 0 || shape >= (int)(sizeof(kShapes) / sizeof(kShapes[0])))
    return bfail(b, TG_INVALID_ARG, "unknown launch shape");
  if (shape != b->shape) {
    drop_graph(b);
    b->shape = shape;
  }
  return TG_OK;
}

tg_status tg_batch_time_steps(tg_batch* b, int steps, double* ms) {
  if (!b || !ms || steps < 1) return bfail(b, TG_INVALID_ARG, "bad argument");
  tg_status st = capture(b);
  if (st != TG_OK) return st;
  cudaEvent_t e0, e1;
  TB_CUDA(b, cudaEventCreate(&e0));
  TB_CUDA(b, cudaEventCreate(&e1));
  TB_CUDA(b, cudaEventRecord(e0, b->stream));
  for (int i = 0; i < steps; ++i) TB_CUDA(b, cudaGraphLaunch(b->graph_exec, b->stream));
  TB_CUDA(b, cudaEventRecord(e1, b->stream));
  if ((st = bsync(b)) != TG_OK) return st;
  float t = 0.0f;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = t / steps;
  return TG_OK;
}

// Autotuner: times `steps` steps of every launch shape from the current state
// (restored after each trial) and keeps the fastest.  ms_out (may be NULL)
// receives the per-shape times in shape order.
tg_status tg_batch_tune(tg_batch* b, int steps, int* shape_out, double* ms_out) {
  if (!b || steps < 1) return bfail(b, TG_INVALID_ARG, "bad argument");
  const int nshape = (int)(sizeof(kShapes) / sizeof(kShapes[0]));
  // save Q[0] and the clocks of every level
  std::vector<void*> saved;
  auto save = [&](const void* src, size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    cudaMemcpyAsync(p, src, bytes, cudaMemcpyDeviceToDevice, b->stream);
    saved.push_back(p);
    return p;
  };
  struct Save { void *q, *el, *cnt, *rch, *bad; };
  std::vector<Save> sv(b->nlev);
  for (int l = 0; l < b->nlev; ++l) {
    const Level& V = b->B.lev[l];
    sv[l].q = save(V.Q[0], (size_t)kQ * V.m.nv * V.P * sizeof(float));
    sv[l].el = save(V.c.elapsed, V.S * sizeof(double));
    sv[l].cnt = save(V.c.counter, V.S * sizeof(int));
    sv[l].rch = save(V.c.reached, V.S * sizeof(int));
    sv[l].bad = save(V.c.bad, V.S * sizeof(int));
    if (!sv[l].q || !sv[l].el || !sv[l].cnt || !sv[l].rch || !sv[l].bad) {
      for (void* p : saved) cudaFree(p);
      return bfail(b, TG_CUDA_ERROR, "no device memory for the tuning snapshot");
    }
  }
  auto restore = [&]() {
    for (int l = 0; l < b->nlev; ++l) {
      const Level& V = b->B.lev[l];
      cudaMemcpyAsync(V.Q[0], sv[l].q, (size_t)kQ * V.m.nv * V.P * sizeof(float), cudaMemcpyDeviceToDevice, b->stream);
      cudaMemcpyAsync(V.c.elapsed, sv[l].el, V.S * sizeof(double), cudaMemcpyDeviceToDevice, b->stream);
      cudaMemcpyAsync(V.c.counter, sv[l].cnt, V.S * sizeof(int), cudaMemcpyDeviceToDevice, b->stream);
      cudaMemcpyAsync(V.c.reached, sv[l].rch, V.S * sizeof(int), cudaMemcpyDeviceToDevice, b->stream);
      cudaMemcpyAsync(V.c.bad, sv[l].bad, V.S * sizeof(int), cudaMemcpyDeviceToDevice, b->stream);
    }
  };
  int best = b->shape;
  double best_ms = 1e300;
  tg_status st = TG_OK;
  for (int i = 0; i < nshape && st == TG_OK; ++i) {
    if ((st = tg_batch_set_shape(b, i)) != TG_OK) break;
    double warm, ms;
    if ((st = tg_batch_time_steps(b, 1, &warm)) != TG_OK) break;
    restore();
    if ((st = tg_batch_time_steps(b, steps, &ms)) != TG_OK) break;
    restore();
    if (ms_out) ms_out[i] = ms;
    if (ms < best_ms) { best_ms = ms; best = i; }
  }
  cudaStreamSynchronize(b->stream);
  for (void* p : saved) cudaFree(p);
  if (st != TG_OK) return st;
  if ((st = tg_batch_set_shape(b, best)) != TG_OK) return st;
  if (shape_out) *shape_out = best;
  return bsync(b);
}

tg_status tg_batch_query(tg_batch* b, int key, double* out) {
  if (!b || !out) return bfail(b, TG_INVALID_ARG, "NULL argument");
  switch (key) {
    case TG_BQ_N_LEVELS: *out = b->nlev; break;
    case TG_BQ_KERNELS_PER_STEP: *out = kernels_per_step(b); break;
    case TG_BQ_DEVICE_BYTES: *out = (double)b->device_bytes; break;
    case TG_BQ_SHAPE: *out = b->shape; break;
    case TG_BQ_SAMPLE_TILE: *out = kShapes[b->shape].st; break;
    case TG_BQ_BLOCK: *out = kShapes[b->shape].bs; break;
    case TG_BQ_N_SHAPES: *out = (double)(sizeof(kShapes) / sizeof(kShapes[0])); break;
    default: return bfail(b, TG_INVALID_ARG, "unknown query key");
  }
  return TG_OK;
}

tg_status tg_batch_stream(tg_batch* b, void** out) {
  if (!b || !out) return bfail(b, TG_INVALID_ARG, "NULL argument");
  *out = (void*)b->stream;
  return TG_OK;
}

}  // extern "C"
