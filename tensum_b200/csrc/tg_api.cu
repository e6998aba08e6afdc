// tg_api.cu -- the C ABI of include/tensum_gpu.h over the device kernels.
//
// Each entry point replaces one FiniteVolume member call of the reference (see
// the header for the mapping).  The handle owns all device memory and one
// stream; whole time steps are captured once into a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <climits>
#include <new>
#include <string>
#include <thread>
#include <deque>
#include <vector>

#include "../../include/tensum_gpu.h"
#include "tg_kernels.cuh"
#include "tg_expr.cuh"
#include "tg_tiles.cuh"
#include "tg_mesh.h"

using namespace tg;

namespace {

thread_local std::string g_last_error;

// Pinned staging for state transfers from and to pageable caller buffers: up to
// kMaxLanes host threads, each with its own stream and two kSlot slots, so the
// host memcpy into one slot overlaps the DMA of the other.  Pinned caller
// buffers bypass it (one cudaMemcpyAsync on the handle's stream).
struct Stager {
  static constexpr int kMaxLanes = 8;
  static constexpr size_t kSlot = size_t(2) << 20;
  int lanes = 0;
  char* slots = nullptr;   // pinned, lanes * 2 * kSlot bytes
  cudaStream_t st[kMaxLanes] = {};
  cudaEvent_t ev[kMaxLanes][2] = {};
  char* slot(int lane, int k) const { return slots + (2 * (size_t)lane + k) * kSlot; }
};

}  // namespace

struct tg_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  HostLayout L;
  Params prm{};
  Control ctl{};
  MeshView mv{};
  StateView sv{};
  TileView tv{};
  double* Pb[3] = {nullptr, nullptr, nullptr};   // rotating state buffers (buffer 0 = current state)
  double* Wb[3] = {nullptr, nullptr, nullptr};
  size_t smem_grad0 = 0, smem_grad1 = 0, smem_flux = 0;
  Scalars* sc = nullptr;       // device
  int* done = nullptr;         // device flag written by k_step_begin
  int* never = nullptr;        // device zero, used by single-phase calls
  double* tinst = nullptr;
  std::vector<void*> allocs;
  std::string err;
  int nblocks_v = 0;
  bool viscous = false;
  bool grads_needed = false;
  cudaGraph_t graph = nullptr;                 // a step that forms its own dt (any state)
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraph_t wgraph = nullptr;                // a step whose dt the previous step formed
  cudaGraphExec_t wgraph_exec = nullptr;
  bool cold = true;                            // the next step may not find dt_next set
  bool w_partial[3] = {false, false, false};   // a step left only V5 in this buffer's W (refresh_w)
  // state transfers: PrimVar records in the caller's order on the device
  double* raw = nullptr;              // 5 * nv doubles
  const int* old_of_new = nullptr;    // device copy of the vertex permutation
  int* bad = nullptr;                 // device flag of k_state_check
  cudaEvent_t raw_ready = nullptr;
  Stager stage;
  // output snapshots (tg_output_begin / tg_output_wait)
  double* snap = nullptr;             // 5 * nv: PrimVar records in the caller's order
  double* snap_grad = nullptr;        // 15 * nv: dE records in the caller's order
  cudaStream_t out_stream = nullptr;
  cudaEvent_t snap_ready = nullptr, out_done = nullptr;
  bool out_pending = false;
  // asynchronous state input (tg_set_state_async): two staging buffers, a copy stream,
  // and the queue of states (slot, start time) the next tg_step / tg_advance takes in order
  double* in_stage[2] = {nullptr, nullptr};
  cudaStream_t in_stream = nullptr;
  cudaEvent_t in_done[2] = {nullptr, nullptr};
  int in_next = 0;
  std::deque<std::pair<int, double>> in_queue;
  bool in_check = false;              // a queued state was taken in: its check is read after the step
  // Monte Carlo moments: per output instance three [nvar][nv] arrays (fm, sm, m2)
  int mom_ninst = 0, mom_extras = 0, mom_nvar = 0;
  double* mom = nullptr;
  double* mom_in = nullptr;   // upload area for a host-side group in tg_moments_merge
  size_t device_bytes = 0;
  int kernels_per_step = 0;
  int kernels_per_flux = 0;
  int n_caller = 0;           // PrimVar records in the caller's state arrays (the whole mesh)
  // domain decomposition (tg_part_create): one partition of a mesh, ghosts filled by the
  // caller's halo exchange (tg_part_pack / tg_part_unpack)
  struct {
    int n_parts = 0, part = 0, n_owned = 0, n_send = 0, n_recv = 0;
    std::vector<int> send_off, recv_off;
    const int* send_idx = nullptr;       // device: local ids of owned vertices, per peer
    const int* recv_idx = nullptr;       // device: local ids of ghosts, per peer
    int cur = 0;                         // state buffer the last flux phase wrote
    int n_frontier = 0;                  // tiles that read ghosts: tile order [0, n_frontier), interior after
    bool norms_pending = false;          // a step ended since the last tg_part_import
    double* out = nullptr;               // device: owned PrimVar records (tg_get_state)
  } part;
};

namespace {

tg_status fail(tg_handle* h, tg_status st, const std::string& msg) {
  if (h) h->err = msg;
  g_last_error = msg;
  return st;
}

#define TG_CUDA(h, call)                                                                             \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      return fail((h), TG_CUDA_ERROR, std::string(#call " failed: ") + cudaGetErrorString(e_));     \
  } while (0)

template <class T>
tg_status dev_upload(tg_handle* h, const std::vector<T>& v, const T** out) {
  void* p = nullptr;
  size_t bytes = std::max<size_t>(1, v.size()) * sizeof(T);
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) return fail(h, TG_CUDA_ERROR, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  h->allocs.push_back(p);
  h->device_bytes += bytes;
  if (!v.empty()) {
    e = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(h, TG_CUDA_ERROR, std::string("cudaMemcpy: ") + cudaGetErrorString(e));
  }
  *out = (const T*)p;
  return TG_OK;
}

template <class T>
tg_status dev_alloc(tg_handle* h, size_t n, T** out) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(T));
  if (e != cudaSuccess) return fail(h, TG_CUDA_ERROR, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  h->allocs.push_back(p);
  h->device_bytes += std::max<size_t>(1, n) * sizeof(T);
  cudaMemset(p, 0, std::max<size_t>(1, n) * sizeof(T));
  *out = (T*)p;
  return TG_OK;
}

inline int nblk(int n) { return (n + kBlock - 1) / kBlock; }

// ---- kernel dispatch over (flux, reconstruction)
typedef void (*BfluxKernel)(Params, MeshView, StateView, const int*);
// Entry points that step or read the whole mesh: a partition handle steps through tg_part_*.
#define TG_WHOLE_MESH(h) \
  if ((h) && (h)->part.n_parts > 0) return fail((h), TG_NOT_SUPPORTED, "a partition handle steps through tg_part_*");

typedef void (*TileFluxKernel)(Params, MeshView, TileView, StateView, Control, Scalars*, int, int, double*, double*,
                               int, int, const int*);

template <int F>
BfluxKernel pick_bflux(int recon) {
  switch (recon) {
    case RECON_FIRST: return k_bflux<F, RECON_FIRST>;
    case RECON_SECOND: return k_bflux<F, RECON_SECOND>;
    case RECON_SECOND_MUSCL: return k_bflux<F, RECON_SECOND_MUSCL>;
    case RECON_VAN_ALBADA: return k_bflux<F, RECON_VAN_ALBADA>;
    case RECON_TVD_MINMOD: return k_bflux<F, RECON_TVD_MINMOD>;
    case RECON_TVB_MINMOD: return k_bflux<F, RECON_TVB_MINMOD>;
    default: return k_bflux<F, RECON_ENO2>;
  }
}
BfluxKernel bflux_kernel(int flux, int recon) {
  switch (flux) {
    case FLUX_TECNO_ROE: return pick_bflux<FLUX_TECNO_ROE>(recon);
    case FLUX_TECNO_RUSANOV: return pick_bflux<FLUX_TECNO_RUSANOV>(recon);
    case FLUX_KEPEC: return k_bflux<FLUX_KEPEC, RECON_FIRST>;
    case FLUX_KEP: return k_bflux<FLUX_KEP, RECON_FIRST>;
    case FLUX_ROE_EC: return k_bflux<FLUX_ROE_EC, RECON_FIRST>;
    default: return k_bflux<FLUX_AVG, RECON_FIRST>;
  }
}

template <int F, int M, bool O>
TileFluxKernel pick_tile(int recon) {
  switch (recon) {
    case RECON_FIRST: return k_tile_flux<F, RECON_FIRST, M, O>;
    case RECON_SECOND: return k_tile_flux<F, RECON_SECOND, M, O>;
    case RECON_SECOND_MUSCL: return k_tile_flux<F, RECON_SECOND_MUSCL, M, O>;
    case RECON_VAN_ALBADA: return k_tile_flux<F, RECON_VAN_ALBADA, M, O>;
    case RECON_TVD_MINMOD: return k_tile_flux<F, RECON_TVD_MINMOD, M, O>;
    case RECON_TVB_MINMOD: return k_tile_flux<F, RECON_TVB_MINMOD, M, O>;
    default: return k_tile_flux<F, RECON_ENO2, M, O>;
  }
}
template <int M, bool O>
TileFluxKernel tile_kernel_m(int flux, int recon) {
  switch (flux) {
    case FLUX_TECNO_ROE: return pick_tile<FLUX_TECNO_ROE, M, O>(recon);
    case FLUX_TECNO_RUSANOV: return pick_tile<FLUX_TECNO_RUSANOV, M, O>(recon);
    case FLUX_KEPEC: return k_tile_flux<FLUX_KEPEC, RECON_FIRST, M, O>;
    case FLUX_KEP: return k_tile_flux<FLUX_KEP, RECON_FIRST, M, O>;
    case FLUX_ROE_EC: return k_tile_flux<FLUX_ROE_EC, RECON_FIRST, M, O>;
    default: return k_tile_flux<FLUX_AVG, RECON_FIRST, M, O>;
  }
}
size_t flux_smem(int flux, int recon, int lmax, int emax, int cmax) {
  const bool grad = recon != RECON_FIRST;
  switch (flux) {
    case FLUX_TECNO_ROE:
      return grad ? tile_flux_smem_t<FLUX_TECNO_ROE, RECON_TVD_MINMOD>(lmax, emax, cmax)
                  : tile_flux_smem_t<FLUX_TECNO_ROE, RECON_FIRST>(lmax, emax, cmax);
    case FLUX_TECNO_RUSANOV:
      return grad ? tile_flux_smem_t<FLUX_TECNO_RUSANOV, RECON_TVD_MINMOD>(lmax, emax, cmax)
                  : tile_flux_smem_t<FLUX_TECNO_RUSANOV, RECON_FIRST>(lmax, emax, cmax);
    case FLUX_KEPEC: return tile_flux_smem_t<FLUX_KEPEC, RECON_FIRST>(lmax, emax, cmax);
    case FLUX_KEP: return tile_flux_smem_t<FLUX_KEP, RECON_FIRST>(lmax, emax, cmax);
    case FLUX_ROE_EC: return tile_flux_smem_t<FLUX_ROE_EC, RECON_FIRST>(lmax, emax, cmax);
    default: return tile_flux_smem_t<FLUX_AVG, RECON_FIRST>(lmax, emax, cmax);
  }
}

// The dynamic shared-memory limit is an attribute of the kernel, shared by every
// handle in the process: it is only ever raised, so a later handle with smaller
// tiles does not lower it below what an earlier handle's launches need.
cudaError_t raise_smem(const void* f, size_t bytes) {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, f);
  if (e != cudaSuccess) return e;
  if ((size_t)a.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

typedef void (*TileGradKernel)(Params, MeshView, TileView, StateView, Scalars*, int, int, const int*, int);
// ord: a partition's launches over its tile order (frontier / interior), whose
// gradient and flux + update kernels are separate instantiations (ORD), so the
// whole-mesh kernels stay exactly as they are
TileGradKernel grad_kernel(bool first, bool grad, bool ord = false) {
  if (first) return grad ? k_tile_grad<true, true> : k_tile_grad<true, false>;
  return ord ? k_tile_grad<false, true, true> : k_tile_grad<false, true>;
}

TileFluxKernel tile_kernel(int flux, int recon, int mode, bool ord = false) {
  if (ord) return tile_kernel_m<MODE_UPDATE, true>(flux, recon);
  return mode == MODE_UPDATE ? tile_kernel_m<MODE_UPDATE, false>(flux, recon)
                             : tile_kernel_m<MODE_RESIDUAL, false>(flux, recon);
}

// state view of buffer b (the three P/W buffers rotate through the stages)
StateView view(const tg_handle* h, int b) {
  StateView v = h->sv;
  v.P = h->Pb[b];
  v.W = h->Wb[b];
  return v;
}

// ---- phases (all enqueue on h->stream; `done` gates work inside graphs)
// Gradients (when `grad`), plus at the first stage dt and U_old.
// At a step's first stage with fuse_dt, the first-stage kernel runs when dt and
// U_old are still to be formed, else a gradient-only launch (warm) takes its place.
// Tiles [base, base + count) of the handle's tile order (all tiles by default).
TileView tiles(const tg_handle* h, int base) {
  TileView v = h->tv;
  v.base = base;
  return v;
}

void enqueue_gradient(tg_handle* h, int b, bool first, bool grad, const int* done, int base = 0, int count = -1) {
  if (!first && !grad) return;
  if (count < 0) count = h->L.ntiles;
  if (count == 0) return;
  const bool ord = h->tv.order != nullptr && !first;   // first-stage passes cover all tiles unordered
  grad_kernel(first, grad, ord)<<<count, kTileThreads, first ? h->smem_grad1 : h->smem_grad0, h->stream>>>(
      h->prm, h->mv, tiles(h, base), view(h, b), h->sc, h->L.lmax, h->L.emax, done, 0);
  if (first && grad && h->prm.fuse_dt)
    grad_kernel(false, true)<<<count, kTileThreads, h->smem_grad0, h->stream>>>(
        h->prm, h->mv, tiles(h, base), view(h, b), h->sc, h->L.lmax, h->L.emax, done, 1);
}

// boundary-face and viscous contributions, gathered by the tiled flux kernel
void enqueue_boundary(tg_handle* h, int b, const int* done) {
  if (h->mv.nb > 0)
    bflux_kernel(h->prm.flux, h->prm.recon)<<<nblk(2 * h->mv.nb), kBlock, 0, h->stream>>>(h->prm, h->mv, view(h, b),
                                                                                            done);
  if (h->viscous) k_viscous<<<nblk(h->mv.nvu), kBlock, 0, h->stream>>>(h->prm, h->mv, view(h, b), done);
}

void enqueue_tile_flux(tg_handle* h, int b, int mode, int r, bool norm, int bout, const int* done, int base = 0,
                       int count = -1) {
  if (count < 0) count = h->L.ntiles;
  if (count == 0) return;
  const bool ord = h->tv.order != nullptr && mode == MODE_UPDATE;
  tile_kernel(h->prm.flux, h->prm.recon, mode, ord)<<<count, kTileThreads, h->smem_flux, h->stream>>>(
      h->prm, h->mv, tiles(h, base), view(h, b), h->ctl, h->sc, r, norm ? 1 : 0, h->Pb[bout], h->Wb[bout], h->L.lmax,
      h->L.emax, done);
}

// Inviscid central-flux steps without strong conditions store only V5 of the entropy
// variables (w3_only in k_tile_flux).  Steps mark the buffers they wrote; before
// gradients are formed outside a step, a marked buffer gets all four back from P.
void mark_steps(tg_handle* h) {
  const bool central = h->prm.flux != FLUX_TECNO_ROE && h->prm.flux != FLUX_TECNO_RUSANOV;
  if (central && h->prm.model == 0 && !h->prm.strong)
    for (int b = 0; b < 3; ++b) h->w_partial[b] = true;
}

void refresh_w(tg_handle* h, int b) {
  if (!h->w_partial[b]) return;
  k_prim2ent<<<nblk(h->mv.nv), kBlock, 0, h->stream>>>(h->prm, h->mv.nv, h->Pb[b], h->Wb[b]);
  h->w_partial[b] = false;
}

int residual_kernels(const tg_handle* h) {
  return (h->mv.nb > 0 ? 1 : 0) + (h->viscous ? 1 : 0) + 1;
}

// compute_residual on buffer 0 (gradient, boundary/viscous terms, tiled fluxes -> R)
void enqueue_residual(tg_handle* h, const int* done) {
  enqueue_gradient(h, 0, false, true, done);
  enqueue_boundary(h, 0, done);
  enqueue_tile_flux(h, 0, MODE_RESIDUAL, 0, false, 0, done);
}

// compute_ssw follows compute_dt in FiniteVolume::solve (src/fv.cc:2282-2285)
void enqueue_ssw(tg_handle* h, const int* done) {
  if (!h->prm.liou) return;
  cudaMemsetAsync(h->sv.ssw, 0, h->mv.nv * sizeof(int), h->stream);
  k_ssw<<<(h->mv.ne + kBlock - 1) / kBlock, kBlock, 0, h->stream>>>(h->prm, h->mv, view(h, 0), done);
}

void enqueue_dt(tg_handle* h, const int* done) {
  if (h->ctl.time_step <= 0.0)
    k_dt<<<nblk(h->mv.nv), kBlock, 0, h->stream>>>(h->prm, h->mv, view(h, 0), h->sc, done);
  k_dt_final<<<1, 1, 0, h->stream>>>(h->ctl, h->sc, done);
  enqueue_ssw(h, done);
}

void enqueue_update(tg_handle* h, int r, bool norm, const int* done) {
  k_update<<<nblk(h->mv.nv), kBlock, 0, h->stream>>>(h->prm, h->mv, view(h, 0), h->ctl, h->sc, r, norm ? 1 : 0, done);
}

void enqueue_norm_final(tg_handle* h, int nblocks, bool use_sc_iter, long long iter, const int* done) {
  k_norm_final<<<1, kBlock, 0, h->stream>>>(h->sv, nblocks, h->mv.nv, h->sc, use_sc_iter ? 1 : 0, iter, done);
}

// One iteration of FiniteVolume::solve's loop on the rotating buffers:
// stage r reads buffer r and writes buffer (r+1)%3, so the step ends in buffer 0.
// The last stage's update also forms the residual norms and ends the iteration
// (its last block).  warm: the previous step's last update formed this step's dt
// and U_old (dt_next set), so the first-stage dt pass and k_dt_final are left out.
void enqueue_step(tg_handle* h, bool warm) {
  k_step_begin<<<1, 1, 0, h->stream>>>(h->ctl, h->sc, h->done, warm ? 1 : 0);
  // stage r reads buffer bin and writes bout: ssprk3 0->1->2->0, rk4 0->1->2->1->0,
  // so a step always ends in buffer 0 and no stage writes the buffer it reads
  const int rk4_in[4] = {0, 1, 2, 1}, rk4_out[4] = {1, 2, 1, 0};
  for (int r = 0; r < h->ctl.n_rks; ++r) {
    const bool first = (r == 0), last = (r == h->ctl.n_rks - 1);
    const int bin = h->ctl.scheme == 1 ? rk4_in[r] : r, bout = h->ctl.scheme == 1 ? rk4_out[r] : (r + 1) % 3;
    if (first && h->ctl.time_step > 0.0) {
      k_store_old<<<nblk(h->mv.nv), kBlock, 0, h->stream>>>(h->prm, h->mv, view(h, 0), h->done);
      enqueue_gradient(h, bin, false, h->grads_needed, h->done);
    } else if (first && warm) {
      enqueue_gradient(h, bin, false, h->grads_needed, h->done);
    } else {
      enqueue_gradient(h, bin, first, h->grads_needed, h->done);   // first stage: + dt, U_old
    }
    if (first && !warm) k_dt_final<<<1, 1, 0, h->stream>>>(h->ctl, h->sc, h->done);
    if (first) enqueue_ssw(h, h->done);
    enqueue_boundary(h, bin, h->done);
    enqueue_tile_flux(h, bin, MODE_UPDATE, r, last, bout, h->done);
    if (h->prm.strong && h->mv.nsb > 0)
      k_strong_bc<<<nblk(h->mv.nsb), kBlock, 0, h->stream>>>(h->mv, h->Pb[bout], h->done);
  }
}

// The captured step to replay: the warm one once the host has seen the previous
// step form dt and U_old for the current state (cold is cleared only then).
cudaGraphExec_t step_graph(const tg_handle* h) {
  return (h->prm.fuse_dt && !h->cold && h->wgraph_exec) ? h->wgraph_exec : h->graph_exec;
}

void drop_graphs(tg_handle* h) {
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  if (h->wgraph_exec) cudaGraphExecDestroy(h->wgraph_exec);
  if (h->wgraph) cudaGraphDestroy(h->wgraph);
  h->graph_exec = h->wgraph_exec = nullptr;
  h->graph = h->wgraph = nullptr;
}

// The state changed outside a captured step: the next step forms dt and U_old itself.
void clear_dt_next(tg_handle* h) {
  cudaMemsetAsync(&h->sc->dt_next, 0, sizeof(int), h->stream);
  h->cold = true;
}

tg_status sync(tg_handle* h) {
  TG_CUDA(h, cudaGetLastError());
  TG_CUDA(h, cudaStreamSynchronize(h->stream));
  return TG_OK;
}

bool host_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// One lane of a staged host->device copy of len bytes.
cudaError_t lane_h2d(const tg_handle* h, int lane, char* dst, const char* src, size_t len) {
  const Stager& S = h->stage;
  cudaError_t e = cudaSetDevice(h->device);
  for (size_t off = 0, k = 0; e == cudaSuccess && off < len; off += Stager::kSlot, ++k) {
    const int s = (int)(k & 1);
    const size_t n = std::min(Stager::kSlot, len - off);
    if (k >= 2 && (e = cudaEventSynchronize(S.ev[lane][s])) != cudaSuccess) break;
    std::memcpy(S.slot(lane, s), src + off, n);
    if ((e = cudaMemcpyAsync(dst + off, S.slot(lane, s), n, cudaMemcpyHostToDevice, S.st[lane])) != cudaSuccess) break;
    e = cudaEventRecord(S.ev[lane][s], S.st[lane]);
  }
  cudaError_t e2 = cudaStreamSynchronize(S.st[lane]);
  return e != cudaSuccess ? e : e2;
}

// One lane of a staged device->host copy; the lane's stream first waits for `ready`.
cudaError_t lane_d2h(const tg_handle* h, int lane, char* dst, const char* src, size_t len, cudaEvent_t ready) {
  const Stager& S = h->stage;
  cudaError_t e = cudaSetDevice(h->device);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(S.st[lane], ready, 0);
  const size_t nk = (len + Stager::kSlot - 1) / Stager::kSlot;
  auto issue = [&](size_t k) {
    const int s = (int)(k & 1);
    const size_t n = std::min(Stager::kSlot, len - k * Stager::kSlot);
    cudaError_t ei = cudaMemcpyAsync(S.slot(lane, s), src + k * Stager::kSlot, n, cudaMemcpyDeviceToHost, S.st[lane]);
    return ei != cudaSuccess ? ei : cudaEventRecord(S.ev[lane][s], S.st[lane]);
  };
  for (size_t k = 0; e == cudaSuccess && k < std::min<size_t>(2, nk); ++k) e = issue(k);
  for (size_t k = 0; e == cudaSuccess && k < nk; ++k) {
    const int s = (int)(k & 1);
    if ((e = cudaEventSynchronize(S.ev[lane][s])) != cudaSuccess) break;
    std::memcpy(dst + k * Stager::kSlot, S.slot(lane, s), std::min(Stager::kSlot, len - k * Stager::kSlot));
    if (k + 2 < nk) e = issue(k + 2);
  }
  cudaError_t e2 = cudaStreamSynchronize(S.st[lane]);
  return e != cudaSuccess ? e : e2;
}

// Splits a staged copy over the lanes (lane 0 on the calling thread).
template <class Lane>
cudaError_t run_lanes(const tg_handle* h, size_t bytes, Lane lane) {
  const int n = (int)std::max<size_t>(1, std::min<size_t>(h->stage.lanes, bytes / (2 * Stager::kSlot)));
  const size_t per = ((bytes + n - 1) / n + 255) & ~size_t(255);
  std::vector<cudaError_t> errs(n, cudaSuccess);
  std::vector<std::thread> th;
  for (int t = 1; t < n; ++t) {
    const size_t off = t * per;
    if (off >= bytes) break;
    th.emplace_back([&, t, off] { errs[t] = lane(t, off, std::min(per, bytes - off)); });
  }
  errs[0] = lane(0, 0, std::min(per, bytes));
  for (auto& x : th) x.join();
  for (cudaError_t e : errs)
    if (e != cudaSuccess) return e;
  return cudaSuccess;
}

// Caller buffer -> h->raw, ordered before the next work on h->stream.
tg_status state_h2d(tg_handle* h, const double* prim, size_t bytes) {
  if (host_pinned(prim)) {
    TG_CUDA(h, cudaMemcpyAsync(h->raw, prim, bytes, cudaMemcpyHostToDevice, h->stream));
    return TG_OK;
  }
  TG_CUDA(h, cudaStreamSynchronize(h->stream));   // h->raw may still be read by an earlier transfer
  const char* src = (const char*)prim;
  char* dst = (char*)h->raw;
  TG_CUDA(h, run_lanes(h, bytes, [&](int t, size_t off, size_t len) { return lane_h2d(h, t, dst + off, src + off, len); }));
  return TG_OK;
}

// h->raw -> caller buffer, after the work enqueued so far on h->stream; returns when the data is in `prim`.
tg_status state_d2h(tg_handle* h, double* prim, size_t bytes) {
  if (host_pinned(prim)) {
    TG_CUDA(h, cudaMemcpyAsync(prim, h->raw, bytes, cudaMemcpyDeviceToHost, h->stream));
    TG_CUDA(h, cudaStreamSynchronize(h->stream));
    return TG_OK;
  }
  TG_CUDA(h, cudaEventRecord(h->raw_ready, h->stream));
  const char* src = (const char*)h->raw;
  char* dst = (char*)prim;
  TG_CUDA(h, run_lanes(h, bytes, [&](int t, size_t off, size_t len) {
    return lane_d2h(h, t, dst + off, src + off, len, h->raw_ready);
  }));
  return TG_OK;
}

tg_status read_scalars(tg_handle* h, Scalars* out) {
  TG_CUDA(h, cudaMemcpyAsync(out, h->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, h->stream));
  return sync(h);
}

// Step bookkeeping of a state that starts at time t0 (FiniteVolume::initialize_sample_run).
Scalars fresh_scalars(const tg_handle* h, double t0) {
  Scalars s;
  std::memset(&s, 0, sizeof(s));
  s.elapsed = t0;
  s.rtotal = 1.0e20;
  s.rtotal0 = 1.0;
  s.counter = 1;
  if (h->ctl.time_mode == 1) {
    double dti = h->ctl.final_time / (h->ctl.ntinst - 1);
    while (s.counter < h->ctl.ntinst - 1 && s.counter * dti <= t0) s.counter++;
  }
  s.dtmin_bits = 0x7ff0000000000000ull;
  s.stop_counter = INT_MAX;
  return s;
}

// The oldest state queued by tg_set_state_async becomes current, in stream order
// after its copy, if k_state_check accepts it (read back by queued_input_refused).
tg_status take_queued_input(tg_handle* h) {
  if (h->in_queue.empty()) return TG_OK;
  const int slot = h->in_queue.front().first;
  const double t0 = h->in_queue.front().second;
  h->in_queue.pop_front();
  const int nv = h->L.nv;
  TG_CUDA(h, cudaStreamWaitEvent(h->stream, h->in_done[slot], 0));
  TG_CUDA(h, cudaMemsetAsync(h->bad, 0, sizeof(int), h->stream));
  k_state_check<<<nblk(nv), kBlock, 0, h->stream>>>(nv, h->in_stage[slot], h->bad);
  k_state_in<<<nblk(nv), kBlock, 0, h->stream>>>(nv, h->in_stage[slot], h->old_of_new, h->bad, h->sv.P);
  k_prim2ent_checked<<<nblk(nv), kBlock, 0, h->stream>>>(h->prm, nv, h->sv.P, h->sv.W, h->bad);
  h->w_partial[0] = false;
  k_scalars_set<<<1, 1, 0, h->stream>>>(h->sc, fresh_scalars(h, t0), h->bad);
  h->in_check = true;
  h->cold = true;
  TG_CUDA(h, cudaGetLastError());
  return TG_OK;
}

tg_status queued_input_refused(tg_handle* h) {
  if (!h->in_check) return TG_OK;
  h->in_check = false;
  int bad = 0;
  TG_CUDA(h, cudaMemcpy(&bad, h->bad, sizeof(int), cudaMemcpyDeviceToHost));
  if (bad) return fail(h, TG_INVALID_ARG, "a state queued by tg_set_state_async was refused (T > 0 and p > 0, "
                                           "src/fv.cc:388-389); the step ran on the previous state");
  return TG_OK;
}

tg_status check_bad(tg_handle* h) {
  Scalars s;
  tg_status st = read_scalars(h, &s);
  if (st != TG_OK) return st;
  if (s.bad) return fail(h, TG_BAD_STATE, "non-finite or non-positive state produced by an update");
  return TG_OK;
}

}  // namespace

tg_status capture_step_graph(tg_handle* h) {
  if (h->graph_exec) return TG_OK;
  for (int w = 0; w < (h->prm.fuse_dt ? 2 : 1); ++w) {
    cudaGraph_t* g = w ? &h->wgraph : &h->graph;
    TG_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_step(h, w == 1);
    cudaError_t e = cudaStreamEndCapture(h->stream, g);
    if (e != cudaSuccess) return fail(h, TG_CUDA_ERROR, std::string("graph capture: ") + cudaGetErrorString(e));
    TG_CUDA(h, cudaGraphInstantiate(w ? &h->wgraph_exec : &h->graph_exec, *g, 0));
  }
  return TG_OK;
}

void enqueue_phase(tg_handle* h, int phase) {
  switch (phase) {
    case TG_PHASE_GRADIENT: enqueue_gradient(h, 0, false, true, h->never); break;
    case TG_PHASE_FLUX:
      enqueue_boundary(h, 0, h->never);
      enqueue_tile_flux(h, 0, MODE_RESIDUAL, 0, false, 0, h->never);
      break;
    case TG_PHASE_UPDATE: enqueue_update(h, 1, false, h->never); break;
    case TG_PHASE_DT: enqueue_dt(h, h->never); break;
    default:
      cudaGraphLaunch(step_graph(h), h->stream);
      mark_steps(h);
      break;
  }
}

// InitialCondition::value (src/ic.h:79-104) at every vertex, on the device, written
// as PrimVar records in the caller's order into the state staging buffer.
__global__ void k_state_expr(int nv, const double* __restrict__ x, const double* __restrict__ y,
                             const int* __restrict__ old_of_new, expr::Field5 f, const double* __restrict__ rnd,
                             int nrnd, double* __restrict__ raw, int* __restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  int e = 0;
  const double xv = x[i], yv = y[i];
  double* q = raw + 5 * (size_t)old_of_new[i];
  q[0] = expr::eval5(f, 0, xv, yv, 0.0, rnd, nrnd, &e);   // temperature
  q[2] = expr::eval5(f, 1, xv, yv, 0.0, rnd, nrnd, &e);   // x velocity
  q[3] = expr::eval5(f, 2, xv, yv, 0.0, rnd, nrnd, &e);   // y velocity
  q[4] = expr::eval5(f, 3, xv, yv, 0.0, rnd, nrnd, &e);   // z velocity
  q[1] = expr::eval5(f, 4, xv, yv, 0.0, rnd, nrnd, &e);   // pressure
  if (e) atomicOr(err, e);
}

// The state in the staging buffer (PrimVar records, caller's order) becomes
// current if every vertex passes the reference's check, with fresh bookkeeping.
tg_status take_raw_state(tg_handle* h, double t0) {
  const int nv = h->L.nv, nc = h->n_caller;   // a partition checks every record, takes its local ones
  tg_status st;
  TG_CUDA(h, cudaMemsetAsync(h->bad, 0, sizeof(int), h->stream));
  k_state_check<<<nblk(nc), kBlock, 0, h->stream>>>(nc, h->raw, h->bad);
  k_state_in<<<nblk(nv), kBlock, 0, h->stream>>>(nv, h->raw, h->old_of_new, h->bad, h->sv.P);
  int bad = 0;
  TG_CUDA(h, cudaMemcpyAsync(&bad, h->bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  if ((st = sync(h)) != TG_OK) return st;
  if (bad) return fail(h, TG_INVALID_ARG, "state needs T > 0 and p > 0 (src/fv.cc:388-389)");
  k_prim2ent<<<nblk(nv), kBlock, 0, h->stream>>>(h->prm, nv, h->sv.P, h->sv.W);
  h->w_partial[0] = false;
  const Scalars s = fresh_scalars(h, t0);
  TG_CUDA(h, cudaMemcpyAsync(h->sc, &s, sizeof(s), cudaMemcpyHostToDevice, h->stream));
  h->cold = true;
  return sync(h);
}

extern "C" {

int tg_abi_version(void) { return TG_ABI_VERSION; }

const char* tg_last_error(const tg_handle* h) {
  if (h && !h->err.empty()) return h->err.c_str();
  return g_last_error.c_str();
}

// tg_create (n_parts = 0) and tg_part_create (partition `part` of n_parts).
static tg_status create_handle(const tg_mesh* mesh, const tg_material* mat, const tg_bc_table* bc,
                               const tg_options* opt, int n_parts, int part, tg_handle** out) {
  if (!out) return fail(nullptr, TG_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (!mesh || !mat || !opt) return fail(nullptr, TG_INVALID_ARG, "mesh, material or options is NULL");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(nullptr, TG_NO_DEVICE, "no CUDA device visible; the GPU path has no CPU fallback");
  // Heun is not offered: the reference's update (src/fv.cc:1681-1690) assigns
  // U = (r/2) U_old - (1 - r/2) dt R after scaling U, which drops U at r = 0,
  // so there is no working reference behaviour to reproduce.
  if (opt->time_scheme != TG_TIME_SSPRK3 && opt->time_scheme != TG_TIME_RK4)
    return fail(nullptr, TG_NOT_SUPPORTED, "the device path runs ssprk3 and rk4 (heuns: see tg_create)");
  if (mat->flux_scheme < 0 || mat->flux_scheme > 5 || mat->reconstruct_scheme < 0 || mat->reconstruct_scheme > 6)
    return fail(nullptr, TG_INVALID_ARG, "unknown flux or reconstruction scheme");
  if (!(mat->gamma > 1.0) || !(mat->gas_const > 0.0)) return fail(nullptr, TG_INVALID_ARG, "gamma must be > 1, gas_const > 0");
  if (opt->time_mode == TG_UNSTEADY && opt->n_time_stamps <= 0)
    return fail(nullptr, TG_INVALID_ARG, "unsteady runs need n_time_stamps > 0");
  if (!(opt->cfl > 0.0) && !(opt->time_step > 0.0)) return fail(nullptr, TG_INVALID_ARG, "cfl or time_step must be > 0");
  // strong conditions reset the state after the last update, so dt could not come from
  // it (fuse_dt) and would need an exchange inside the step; the Liou switch of a ghost
  // depends on edges the partition does not hold
  if (n_parts > 0 && (opt->bc_strong || (opt->liou_fix && mat->flux_scheme == FLUX_TECNO_ROE)))
    return fail(nullptr, TG_NOT_SUPPORTED, "partitioned runs use weak boundary conditions and no Liou fix");

  tg_handle* h = new (std::nothrow) tg_handle();
  if (!h) return fail(nullptr, TG_INVALID_ARG, "out of host memory");
  cudaGetDevice(&h->device);
  h->viscous = mat->model == 1;
  std::string msg = build_layout(*mesh, bc, h->viscous, h->L);
  if (!msg.empty()) {
    delete h;
    return fail(nullptr, TG_INVALID_ARG, msg);
  }
  h->n_caller = h->L.nv;
  PartPlan plan;
  if (n_parts > 0) {
    HostLayout G = std::move(h->L);
    msg = plan_partition(G, n_parts, part, plan);
    if (msg.empty()) msg = restrict_layout(G, plan, h->L);
    if (!msg.empty()) {
      delete h;
      return fail(nullptr, TG_INVALID_ARG, msg);
    }
  }
  msg = build_tiles(h->L, TG_TILE_OWNED, TG_TILE_LCAP, TG_TILE_ECAP);
  if (!msg.empty()) {
    delete h;
    return fail(nullptr, TG_INVALID_ARG, msg);
  }
  const HostLayout& L = h->L;
  h->grads_needed = h->viscous || ((mat->flux_scheme == FLUX_TECNO_ROE || mat->flux_scheme == FLUX_TECNO_RUSANOV) &&
                                   mat->reconstruct_scheme != RECON_FIRST);

  Params& k = h->prm;
  k.gamma = mat->gamma; k.R = mat->gas_const; k.Cp = mat->gamma * mat->gas_const / (mat->gamma - 1.0);
  k.sqrt_gm1 = std::sqrt(mat->gamma - 1.0);
  k.inv_gamma = 1.0 / mat->gamma;
  k.inv_gm1 = 1.0 / (mat->gamma - 1.0);
  k.gp1_gm1 = (mat->gamma + 1.0) / (mat->gamma - 1.0);
  k.prandtl = mat->prandtl; k.mu_ref = mat->mu_ref; k.T0 = mat->T_0; k.Tref = mat->T_ref; k.omega = mat->omega;
  k.ev_alpha = mat->ev_mod_alpha; k.ev_beta = mat->ev_mod_beta; k.tvbM = mat->tvb_minmod_coef; k.cfl = opt->cfl;
  k.model = mat->model; k.flux = mat->flux_scheme; k.mu_model = mat->mu_model; k.recon = mat->reconstruct_scheme;
  k.nd = mat->nd_active; k.visc = mat->visc_active; k.heat = mat->heat_active;
  k.liou = (opt->liou_fix && mat->flux_scheme == FLUX_TECNO_ROE) ? 1 : 0;
  k.strong = opt->bc_strong ? 1 : 0;
  // strong conditions change the state after the last update; a fixed time step needs no dt
  k.fuse_dt = (!k.strong && opt->time_step <= 0.0) ? 1 : 0;
  k.axi = h->L.axi ? 1 : 0;

  tg_status st;
#define UP(vec, field) \
  if ((st = dev_upload(h, L.vec, &h->mv.field)) != TG_OK) { tg_destroy(h); return st; }
  h->mv.nv = L.nv; h->mv.ne = L.ne; h->mv.nb = L.nb; h->mv.nvu = L.nvu; h->mv.n_int_cells = L.n_int_cells;
  UP(dcarea, dcarea) UP(inv6mc, inv6mc) UP(pweight, pweight)
  UP(e_a, e_a) UP(e_b, e_b) UP(e_nx, e_nx) UP(e_ny, e_ny) UP(e_dx, e_dx) UP(e_dy, e_dy)
  UP(e_g0x, e_g0x) UP(e_g0y, e_g0y) UP(e_g1x, e_g1x) UP(e_g1y, e_g1y)
  UP(ce_off, ce_off) UP(ce_ent, ce_ent) UP(cb_off, cb_off) UP(cb_ent, cb_ent)
  UP(b_v0, b_v0) UP(b_v1, b_v1) UP(b_kind, b_kind) UP(b_adiab, b_adiab) UP(b_cell, b_cell)
  UP(b_nx, b_nx) UP(b_ny, b_ny) UP(b_val, b_val)
  UP(bf_face_nx, bf_face_nx) UP(bf_face_ny, bf_face_ny) UP(bf_face_v0, bf_face_v0) UP(bf_face_v1, bf_face_v1)
  UP(u_cell, u_cell) UP(c_v, c_v) UP(c_n, c_n) UP(c_inv2a, c_inv2a)
  UP(c_bf_off, c_bf_off) UP(c_bf, c_bf) UP(c_nbr_off, c_nbr_off) UP(c_nbr, c_nbr)
  UP(v_r, v_r) UP(u_r, u_r)
  {
    // bc_scheme strong: which vertices a condition resets (slip, no-slip, pressure,
    // inlet) and in which face order, and which lie on no-slip faces
    std::vector<int> sflag(L.nv, 0), sb_v, sb_off(1, 0), sb_ent;
    std::vector<std::vector<int>> per(L.nv);
    for (int d = 0; d < L.nb; ++d) {
      const int kind = L.b_kind[d];
      const bool resets = kind == BC_SLIP || kind == BC_NOSLIP || kind == BC_PRESSURE || kind == BC_INLET;
      for (int slot = 0; slot < 2; ++slot) {
        const int v = slot ? L.b_v1[d] : L.b_v0[d];
        if (resets) { per[v].push_back((d << 1) | slot); sflag[v] |= 1; }
        if (kind == BC_NOSLIP) sflag[v] |= 2;
      }
    }
    for (int v = 0; v < L.nv; ++v) {
      if (per[v].empty()) continue;
      sb_v.push_back(v);
      sb_ent.insert(sb_ent.end(), per[v].begin(), per[v].end());
      sb_off.push_back((int)sb_ent.size());
    }
    h->mv.nsb = opt->bc_strong ? (int)sb_v.size() : 0;
    if ((st = dev_upload(h, sflag, &h->mv.sflag)) != TG_OK) { tg_destroy(h); return st; }
    if ((st = dev_upload(h, sb_v, &h->mv.sb_v)) != TG_OK) { tg_destroy(h); return st; }
    if ((st = dev_upload(h, sb_off, &h->mv.sb_off)) != TG_OK) { tg_destroy(h); return st; }
    if ((st = dev_upload(h, sb_ent, &h->mv.sb_ent)) != TG_OK) { tg_destroy(h); return st; }
  }
#undef UP
#define UPT(vec, field) \
  if ((st = dev_upload(h, L.vec, &h->tv.field)) != TG_OK) { tg_destroy(h); return st; }
  UPT(t_vbeg, vbeg) UPT(t_loff, loff) UPT(t_eoff, eoff) UPT(lv, lv) UPT(te_ab, ab)
  UPT(te_nx, nx) UPT(te_ny, ny) UPT(te_g0x, g0x) UPT(te_g0y, g0y) UPT(te_g1x, g1x) UPT(te_g1y, g1y)
  UPT(cv_off, cv_off) UPT(cv_ent, cv_ent) UPT(x, x) UPT(y, y) UPT(te_ux, ux) UPT(te_uy, uy) UPT(te_ar, ar)
  UPT(te_r, r)
#undef UPT
  h->tv.order = nullptr;
  h->tv.base = 0;
  h->tv.total = L.ntiles;
  const size_t nv = L.nv;
  h->nblocks_v = nblk(L.nv);
#define AL(field, n) \
  if ((st = dev_alloc(h, (n), &h->sv.field)) != TG_OK) { tg_destroy(h); return st; }
  AL(P, 4 * nv) AL(W, 4 * nv) AL(G, 8 * nv) AL(R, 4 * nv) AL(Uold, 4 * nv) AL(dt, nv)
  AL(Fb, 8 * (size_t)L.nb) AL(Fv, 9 * (size_t)L.nvu) AL(Fvb, 3 * (size_t)L.nb)
  AL(part, 4 * (size_t)std::max(h->nblocks_v, L.ntiles)) AL(R2, 4 * nv) AL(ssw, nv)
#undef AL
  h->Pb[0] = h->sv.P;
  h->Wb[0] = h->sv.W;
  for (int b = 1; b < 3; ++b) {
    if ((st = dev_alloc(h, 4 * nv, &h->Pb[b])) != TG_OK) { tg_destroy(h); return st; }
    if ((st = dev_alloc(h, 4 * nv, &h->Wb[b])) != TG_OK) { tg_destroy(h); return st; }
  }
  h->smem_grad0 = tile_grad_smem(L.lmax, L.emax, L.cmax, false);
  h->smem_grad1 = tile_grad_smem(L.lmax, L.emax, L.cmax, true);
  h->smem_flux = flux_smem(mat->flux_scheme, mat->reconstruct_scheme, L.lmax, L.emax, L.cmax);
  {
    cudaError_t ea = raise_smem((const void*)grad_kernel(true, true), h->smem_grad1);
    cudaError_t ea2 = raise_smem((const void*)grad_kernel(true, false), h->smem_grad1);
    cudaError_t eb = raise_smem((const void*)grad_kernel(false, true), h->smem_grad0);
    cudaError_t ec = raise_smem((const void*)tile_kernel(mat->flux_scheme, mat->reconstruct_scheme, MODE_UPDATE),
                                h->smem_flux);
    cudaError_t ed = raise_smem((const void*)tile_kernel(mat->flux_scheme, mat->reconstruct_scheme, MODE_RESIDUAL),
                                h->smem_flux);
    if (ea != cudaSuccess || ea2 != cudaSuccess || eb != cudaSuccess || ec != cudaSuccess || ed != cudaSuccess) {
      tg_destroy(h);
      return fail(nullptr, TG_CUDA_ERROR, "tile kernels need more shared memory than the device allows");
    }
  }
  if ((st = dev_alloc(h, 1, &h->sc)) != TG_OK) { tg_destroy(h); return st; }
  if ((st = dev_alloc(h, 1, &h->done)) != TG_OK) { tg_destroy(h); return st; }
  if ((st = dev_alloc(h, 1, &h->never)) != TG_OK) { tg_destroy(h); return st; }

  // output time instances (src/fv.cc:52-62)
  std::vector<double> ti;
  if (opt->time_mode == TG_UNSTEADY) {
    double dti = opt->final_time / opt->n_time_stamps;
    for (int i = 0; i <= opt->n_time_stamps; ++i) ti.push_back(i * dti);
  } else {
    ti.assign(2, 0.0);
  }
  const double* tip = nullptr;
  if ((st = dev_upload(h, ti, &tip)) != TG_OK) { tg_destroy(h); return st; }
  Control& c = h->ctl;
  c.time_mode = opt->time_mode; c.n_rks = opt->time_scheme == TG_TIME_RK4 ? 4 : 3;
  c.scheme = opt->time_scheme == TG_TIME_RK4 ? 1 : 0;
  c.ntinst = (int)ti.size(); c.time_step = opt->time_step;
  c.min_residue = opt->min_residue; c.max_iter = opt->max_iter; c.final_time = opt->final_time; c.tinst = tip;

  h->kernels_per_flux = residual_kernels(h);
  // launches of a replayed step: step_begin + gradient passes + per stage (boundary,
  // viscous, tiled flux; the last also forms the norms and ends the step) + Liou /
  // strong-condition kernels; a step that forms its own dt adds the first-stage dt
  // pass (and its gradient-only twin) and dt_final, a fixed time step store_old.
  // The count is that of the steady state: warm steps when the next dt is fused.
  const int tail = (k.liou ? 1 : 0) + (k.strong && h->mv.nsb > 0 ? c.n_rks : 0) + c.n_rks * residual_kernels(h);
  const int grads = h->grads_needed ? c.n_rks : 0;
  if (k.fuse_dt) h->kernels_per_step = 1 + grads + tail;
  else if (c.time_step > 0.0) h->kernels_per_step = 1 + 1 + grads + 1 + tail;
  else h->kernels_per_step = 1 + (h->grads_needed ? c.n_rks : 1) + 1 + tail;
  if ((st = dev_alloc(h, 5 * (size_t)h->n_caller, &h->raw)) != TG_OK) { tg_destroy(h); return st; }
  if ((st = dev_alloc(h, 1, &h->bad)) != TG_OK) { tg_destroy(h); return st; }
  if ((st = dev_upload(h, L.old_of_new, &h->old_of_new)) != TG_OK) { tg_destroy(h); return st; }
  {
    Stager& S = h->stage;
    const size_t bytes = 5 * (size_t)h->n_caller * sizeof(double);
    S.lanes = (int)std::max<size_t>(1, std::min<size_t>(Stager::kMaxLanes, bytes / (2 * Stager::kSlot)));
    cudaError_t ep = cudaMallocHost((void**)&S.slots, 2 * (size_t)S.lanes * Stager::kSlot);
    for (int t = 0; t < S.lanes && ep == cudaSuccess; ++t) {
      ep = cudaStreamCreateWithFlags(&S.st[t], cudaStreamNonBlocking);
      for (int k = 0; k < 2 && ep == cudaSuccess; ++k) ep = cudaEventCreateWithFlags(&S.ev[t][k], cudaEventDisableTiming);
    }
    if (ep == cudaSuccess) ep = cudaEventCreateWithFlags(&h->raw_ready, cudaEventDisableTiming);
    if (ep != cudaSuccess) { tg_destroy(h); return fail(nullptr, TG_CUDA_ERROR, cudaGetErrorString(ep)); }
  }
  if (n_parts > 0) {
    auto& P = h->part;
    P.n_parts = n_parts; P.part = part; P.n_owned = plan.n_owned;
    P.send_off = plan.send_off; P.recv_off = plan.recv_off;
    P.n_send = (int)plan.send_idx.size(); P.n_recv = (int)plan.recv_idx.size();
    if ((st = dev_upload(h, plan.send_idx, &P.send_idx)) != TG_OK) { tg_destroy(h); return st; }
    if ((st = dev_upload(h, plan.recv_idx, &P.recv_idx)) != TG_OK) { tg_destroy(h); return st; }
    if ((st = dev_alloc(h, 5 * (size_t)std::max(1, P.n_owned), &P.out)) != TG_OK) { tg_destroy(h); return st; }
    // frontier tiles (some local vertex is a ghost) first, then the interior ones, so a
    // driver can run the interior while a halo exchange is in flight
    std::vector<int> order, interior;
    for (int t = 0; t < L.ntiles; ++t) {
      bool ghost = false;
      for (int i = L.t_loff[t]; i < L.t_loff[t + 1] && !ghost; ++i) ghost = L.lv[i] >= plan.n_owned;
      (ghost ? order : interior).push_back(t);
    }
    P.n_frontier = (int)order.size();
    order.insert(order.end(), interior.begin(), interior.end());
    if ((st = dev_upload(h, order, &h->tv.order)) != TG_OK) { tg_destroy(h); return st; }
    if (raise_smem((const void*)grad_kernel(false, true, true), h->smem_grad0) != cudaSuccess ||
        raise_smem((const void*)tile_kernel(mat->flux_scheme, mat->reconstruct_scheme, MODE_UPDATE, true),
                   h->smem_flux) != cudaSuccess) {
      tg_destroy(h);
      return fail(nullptr, TG_CUDA_ERROR, "tile kernels need more shared memory than the device allows");
    }
    c.part = 1;
  }
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { tg_destroy(h); return fail(nullptr, TG_CUDA_ERROR, cudaGetErrorString(e)); }
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) { tg_destroy(h); return fail(nullptr, TG_CUDA_ERROR, cudaGetErrorString(e)); }
  *out = h;
  return TG_OK;
}

tg_status tg_create(const tg_mesh* mesh, const tg_material* mat, const tg_bc_table* bc, const tg_options* opt,
                    tg_handle** out) {
  return create_handle(mesh, mat, bc, opt, 0, 0, out);
}

tg_status tg_destroy(tg_handle* h) {
  if (!h) return TG_OK;
  drop_graphs(h);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (void* p : h->allocs) cudaFree(p);
  if (h->mom) cudaFree(h->mom);
  if (h->mom_in) cudaFree(h->mom_in);
  for (int t = 0; t < Stager::kMaxLanes; ++t) {
    if (h->stage.st[t]) cudaStreamSynchronize(h->stage.st[t]);
    for (int k = 0; k < 2; ++k)
      if (h->stage.ev[t][k]) cudaEventDestroy(h->stage.ev[t][k]);
    if (h->stage.st[t]) cudaStreamDestroy(h->stage.st[t]);
  }
  if (h->stage.slots) cudaFreeHost(h->stage.slots);
  if (h->raw_ready) cudaEventDestroy(h->raw_ready);
  if (h->out_stream) cudaStreamSynchronize(h->out_stream);
  if (h->in_stream) cudaStreamSynchronize(h->in_stream);
  for (int k = 0; k < 2; ++k)
    if (h->in_done[k]) cudaEventDestroy(h->in_done[k]);
  if (h->in_stream) cudaStreamDestroy(h->in_stream);
  if (h->snap_ready) cudaEventDestroy(h->snap_ready);
  if (h->out_done) cudaEventDestroy(h->out_done);
  if (h->out_stream) cudaStreamDestroy(h->out_stream);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return TG_OK;
}

tg_status tg_set_state(tg_handle* h, const double* prim, int n_vertex, double t0) {
  if (!h || !prim) return fail(h, TG_INVALID_ARG, "NULL argument");
  if (n_vertex != h->n_caller) return fail(h, TG_INVALID_ARG, "n_vertex does not match the mesh");
  if (h->in_stream) TG_CUDA(h, cudaStreamSynchronize(h->in_stream));
  h->in_queue.clear();                 // states queued by tg_set_state_async are dropped
  tg_status st = state_h2d(h, prim, 5 * (size_t)h->n_caller * sizeof(double));
  if (st != TG_OK) return st;
  h->part.cur = 0;
  h->part.norms_pending = false;
  return take_raw_state(h, t0);
}

tg_status tg_set_state_expr(tg_handle* h, const tg_expr* const* fields, const double* rnd, int n_rnd, double t0) {
  TG_WHOLE_MESH(h)
  if (!h || !fields) return fail(h, TG_INVALID_ARG, "NULL argument");
  for (int c = 0; c < 5; ++c)
    if (c != 3 && !fields[c]) return fail(h, TG_INVALID_ARG, "temperature, velocity and pressure expressions are needed");
  if (n_rnd < 0 || (n_rnd > 0 && !rnd)) return fail(h, TG_INVALID_ARG, "bad random numbers");
  if (h->in_stream) TG_CUDA(h, cudaStreamSynchronize(h->in_stream));
  h->in_queue.clear();
  std::vector<int> code, off;
  std::vector<double> k;
  expr::pack5(fields, nullptr, code, off, k);
  int *dcode = nullptr, *doff = nullptr, *derr = nullptr;
  double *dk = nullptr, *drnd = nullptr;
  cudaError_t e = cudaMalloc((void**)&dcode, code.size() * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void**)&doff, off.size() * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void**)&dk, std::max<size_t>(1, k.size()) * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&drnd, std::max(1, n_rnd) * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&derr, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyAsync(dcode, code.data(), code.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(doff, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess && !k.empty()) e = cudaMemcpyAsync(dk, k.data(), k.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess && n_rnd > 0) e = cudaMemcpyAsync(drnd, rnd, n_rnd * sizeof(double), cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(derr, 0, sizeof(int), h->stream);
  int err = 0;
  if (e == cudaSuccess) {
    const int nv = h->L.nv;
    k_state_expr<<<nblk(nv), kBlock, 0, h->stream>>>(nv, h->tv.x, h->tv.y, h->old_of_new, expr::Field5{dcode, doff, dk},
                                                     drnd, n_rnd, h->raw, derr);
    e = cudaMemcpyAsync(&err, derr, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  }
  cudaFree(dcode); cudaFree(doff); cudaFree(dk); cudaFree(drnd); cudaFree(derr);
  if (e != cudaSuccess) return fail(h, TG_CUDA_ERROR, cudaGetErrorString(e));
  if (err) return fail(h, TG_INVALID_ARG, "pert: unknown type or random-number index out of range");
  return take_raw_state(h, t0);
}


tg_status tg_set_state_async(tg_handle* h, const double* prim, int n_vertex, double t0) {
  TG_WHOLE_MESH(h)
  if (!h || !prim) return fail(h, TG_INVALID_ARG, "NULL argument");
  if (n_vertex != h->L.nv) return fail(h, TG_INVALID_ARG, "n_vertex does not match the mesh");
  if (!host_pinned(prim)) return fail(h, TG_INVALID_ARG, "tg_set_state_async copies from pinned host memory");
  if (h->in_queue.size() >= 2) return fail(h, TG_INVALID_ARG, "two states are queued already; step first");
  const size_t bytes = 5 * (size_t)h->L.nv * sizeof(double);
  tg_status st;
  if (!h->in_stream) {
    for (int k = 0; k < 2; ++k)
      if ((st = dev_alloc(h, 5 * (size_t)h->L.nv, &h->in_stage[k])) != TG_OK) return st;
    TG_CUDA(h, cudaStreamCreateWithFlags(&h->in_stream, cudaStreamNonBlocking));
    for (int k = 0; k < 2; ++k) TG_CUDA(h, cudaEventCreateWithFlags(&h->in_done[k], cudaEventDisableTiming));
  }
  // a slot is rewritten only after the step that took its previous state in has returned
  const int slot = h->in_next;
  h->in_next ^= 1;
  TG_CUDA(h, cudaMemcpyAsync(h->in_stage[slot], prim, bytes, cudaMemcpyHostToDevice, h->in_stream));
  TG_CUDA(h, cudaEventRecord(h->in_done[slot], h->in_stream));
  h->in_queue.emplace_back(slot, t0);
  return TG_OK;
}

tg_status tg_get_state(tg_handle* h, double* prim, int n_vertex) {
  if (!h || !prim) return fail(h, TG_INVALID_ARG, "NULL argument");
  if (n_vertex != h->n_caller) return fail(h, TG_INVALID_ARG, "n_vertex does not match the mesh");
  if (h->part.n_parts > 0) {
    // a partition writes the records of the vertices it owns and leaves the others
    const int n = h->part.n_owned;
    std::vector<double> rec(5 * (size_t)n);
    k_part_state_out<<<nblk(std::max(1, n)), kBlock, 0, h->stream>>>(n, h->L.nv, h->Pb[h->part.cur], h->part.out);
    TG_CUDA(h, cudaGetLastError());
    TG_CUDA(h, cudaMemcpyAsync(rec.data(), h->part.out, rec.size() * sizeof(double), cudaMemcpyDeviceToHost,
                               h->stream));
    tg_status st = sync(h);
    if (st != TG_OK) return st;
    for (int i = 0; i < n; ++i) std::memcpy(prim + 5 * (size_t)h->L.old_of_new[i], &rec[5 * (size_t)i], 5 * sizeof(double));
    return TG_OK;
  }
  const int nv = h->L.nv;
  k_state_out<<<nblk(nv), kBlock, 0, h->stream>>>(nv, h->sv.P, h->old_of_new, h->raw);
  TG_CUDA(h, cudaGetLastError());
  return state_d2h(h, prim, 5 * (size_t)nv * sizeof(double));
}

tg_status tg_store_conserved_old(tg_handle* h) {
  TG_WHOLE_MESH(h)
  if (!h) return fail(h, TG_INVALID_ARG, "NULL handle");
  k_store_old<<<nblk(h->mv.nv), kBlock, 0, h->stream>>>(h->prm, h->mv, view(h, 0), h->never);
  return sync(h);
}

tg_status tg_compute_dt(tg_handle* h, double* dt_global_out, double* dt_out) {
  TG_WHOLE_MESH(h)
  if (!h) return fail(h, TG_INVALID_ARG, "NULL handle");
  unsigned long long inf = 0x7ff0000000000000ull;
  TG_CUDA(h, cudaMemcpyAsync(&h->sc->dtmin_bits, &inf, sizeof(inf), cudaMemcpyHostToDevice, h->stream));
  enqueue_dt(h, h->never);
  Scalars s;
  tg_status st = read_scalars(h, &s);
  if (st != TG_OK) return st;
  if (dt_global_out) *dt_global_out = s.dt_global;
  if (dt_out) {
    const int nv = h->L.nv;
    std::vector<double> d(nv);
    if (h->ctl.time_mode == 1 || h->ctl.time_step > 0.0) {
      for (int i = 0; i < nv; ++i) dt_out[i] = s.dt_global;
    } else {
      TG_CUDA(h, cudaMemcpy(d.data(), h->sv.dt, nv * sizeof(double), cudaMemcpyDeviceToHost));
      for (int i = 0; i < nv; ++i) dt_out[h->L.old_of_new[i]] = d[i];
    }
  }
  return TG_OK;
}

static tg_status copy_grad_out(tg_handle* h, double* dE_out) {
  const int nv = h->L.nv;
  std::vector<double> g(8 * (size_t)nv);
  TG_CUDA(h, cudaMemcpy(g.data(), h->sv.G, g.size() * sizeof(double), cudaMemcpyDeviceToHost));
  static const int var_of[4] = {0, 1, 2, 4};
  for (int i = 0; i < nv; ++i) {
    double* d = dE_out + 15 * (size_t)h->L.old_of_new[i];
    for (int q = 0; q < 15; ++q) d[q] = 0.0;
    for (int c = 0; c < 4; ++c) {
      d[3 * var_of[c]] = g[(2 * c) * (size_t)nv + i];
      d[3 * var_of[c] + 1] = g[(2 * c + 1) * (size_t)nv + i];
    }
  }
  return TG_OK;
}

tg_status tg_gradients(tg_handle* h, double* dE_out) {
  TG_WHOLE_MESH(h)
  if (!h) return fail(h, TG_INVALID_ARG, "NULL handle");
  refresh_w(h, 0);
  enqueue_gradient(h, 0, false, true, h->never);
  tg_status st = sync(h);
  if (st != TG_OK || !dE_out) return st;
  return copy_grad_out(h, dE_out);
}

tg_status tg_residual(tg_handle* h, double* res_out) {
  TG_WHOLE_MESH(h)
  if (!h) return fail(h, TG_INVALID_ARG, "NULL handle");
  enqueue_residual(h, h->never);
  tg_status st = sync(h);
  if (st != TG_OK || !res_out) return st;
  const int nv = h->L.nv;
  std::vector<double> r(4 * (size_t)nv);
  TG_CUDA(h, cudaMemcpy(r.data(), h->sv.R, r.size() * sizeof(double), cudaMemcpyDeviceToHost));
  for (int i = 0; i < nv; ++i) {
    double* d = res_out + 5 * (size_t)h->L.old_of_new[i];
    d[0] = r[i]; d[1] = r[nv + i]; d[2] = r[2 * (size_t)nv + i]; d[3] = 0.0; d[4] = r[3 * (size_t)nv + i];
  }
  return TG_OK;
}

tg_status tg_update(tg_handle* h, int r) {
  TG_WHOLE_MESH(h)
  if (!h) return fail(h, TG_INVALID_ARG, "NULL handle");
  if (r < 0 || r >= h->ctl.n_rks) return fail(h, TG_INVALID_ARG, "stage index out of range for the time scheme");
  enqueue_update(h, r, false, h->never);
  h->w_partial[0] = false;                   // k_update stores all four entropy variables
  if (h->prm.strong && h->mv.nsb > 0)
    k_strong_bc<<<nblk(h->mv.nsb), kBlock, 0, h->stream>>>(h->mv, h->sv.P, h->never);
  clear_dt_next(h);
  tg_status st = sync(h);
  if (st != TG_OK) return st;
  return check_bad(h);
}

tg_status tg_residual_norm(tg_handle* h, long iter, double* out6) {
  TG_WHOLE_MESH(h)
  if (!h) return fail(h, TG_INVALID_ARG, "NULL handle");
  if (h->prm.strong) k_strong_zero_res<<<h->nblocks_v, kBlock, 0, h->stream>>>(h->mv, h->sv);
  k_norm_part<<<h->nblocks_v, kBlock, 0, h->stream>>>(h->mv, h->sv, h->never);
  enqueue_norm_final(h, h->nblocks_v, false, iter, h->never);
  Scalars s;
  tg_status st = read_scalars(h, &s);
  if (st != TG_OK) return st;
  if (out6) {
    out6[0] = s.rnorm[0]; out6[1] = s.rnorm[1]; out6[2] = s.rnorm[2]; out6[3] = s.rnorm[3];
    out6[4] = s.rtotal; out6[5] = s.rtotal0;
  }
  return TG_OK;
}

tg_status tg_end_step(tg_handle* h, double* info4) {
  TG_WHOLE_MESH(h)
  if (!h) return fail(h, TG_INVALID_ARG, "NULL handle");
  k_step_end<<<1, 1, 0, h->stream>>>(h->ctl, h->sc, h->never);
  Scalars s;
  tg_status st = read_scalars(h, &s);
  if (st != TG_OK) return st;
  if (info4) { info4[0] = s.elapsed; info4[1] = s.dt_global; info4[2] = s.rtotal; info4[3] = (double)s.iter; }
  return TG_OK;
}

tg_status tg_step(tg_handle* h, int n_steps, double* info4) {
  TG_WHOLE_MESH(h)
  if (!h) return fail(h, TG_INVALID_ARG, "NULL handle");
  if (n_steps < 0) return fail(h, TG_INVALID_ARG, "n_steps < 0");
  tg_status st = capture_step_graph(h);
  if (st != TG_OK) return st;
  if ((st = take_queued_input(h)) != TG_OK) return st;
  const cudaGraphExec_t g = step_graph(h);
  for (int i = 0; i < n_steps; ++i) TG_CUDA(h, cudaGraphLaunch(g, h->stream));
  if (n_steps > 0) mark_steps(h);
  Scalars s;
  st = read_scalars(h, &s);
  if (st != TG_OK) return st;
  h->cold = !s.dt_next;
  if ((st = queued_input_refused(h)) != TG_OK) return st;
  if (info4) { info4[0] = s.elapsed; info4[1] = s.dt_global; info4[2] = s.rtotal; info4[3] = (double)s.iter; }
  if (s.bad) return fail(h, TG_BAD_STATE, "non-finite or non-positive state produced by an update");
  return TG_OK;
}

}  // extern "C"

// ---- output-time stepping and Monte Carlo moments

namespace {

// The solve loop's continuation test (src/fv.cc:2273-2275) on the host copy of the scalars.
bool run_over(const tg_handle* h, const Scalars& s) {
  const bool go = s.rtotal > h->ctl.min_residue && (h->ctl.time_mode == 1 || s.iter < h->ctl.max_iter) &&
                  s.elapsed < h->ctl.final_time;
  return !go;
}

double* mom_array(tg_handle* h, int instance, int which) {
  return h->mom + ((size_t)instance * 3 + which) * (size_t)h->mom_nvar * h->L.nv;
}

tg_status mom_check(tg_handle* h, int instance) {
  if (!h) return fail(h, TG_INVALID_ARG, "NULL handle");
  if (!h->mom) return fail(h, TG_INVALID_ARG, "tg_moments_init has not been called");
  if (instance < 0 || instance >= h->mom_ninst) return fail(h, TG_INVALID_ARG, "output instance out of range");
  return TG_OK;
}

}  // namespace

extern "C" {

tg_status tg_advance(tg_handle* h, int instance, long max_steps, double* info5) {
  TG_WHOLE_MESH(h)
  if (!h) return fail(h, TG_INVALID_ARG, "NULL handle");
  if (max_steps < 0) return fail(h, TG_INVALID_ARG, "max_steps < 0");
  tg_status st = capture_step_graph(h);
  if (st != TG_OK) return st;
  if ((st = take_queued_input(h)) != TG_OK) return st;
  int stop = instance;
  TG_CUDA(h, cudaMemcpyAsync(&h->sc->stop_counter, &stop, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  Scalars s;
  if ((st = read_scalars(h, &s)) != TG_OK) return st;
  if ((st = queued_input_refused(h)) != TG_OK) return st;
  long launched = 0;
  while (launched < max_steps && !s.bad && s.counter <= instance && !run_over(h, s)) {
    const long chunk = std::min<long>(16, max_steps - launched);
    const cudaGraphExec_t g = step_graph(h);
    for (long i = 0; i < chunk; ++i) TG_CUDA(h, cudaGraphLaunch(g, h->stream));
    mark_steps(h);
    launched += chunk;
    if ((st = read_scalars(h, &s)) != TG_OK) return st;
    h->cold = !s.dt_next;
  }
  stop = INT_MAX;
  TG_CUDA(h, cudaMemcpyAsync(&h->sc->stop_counter, &stop, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  if ((st = sync(h)) != TG_OK) return st;
  if (info5) {
    info5[0] = s.elapsed; info5[1] = s.dt_global; info5[2] = s.rtotal; info5[3] = (double)s.iter;
    info5[4] = (double)s.counter;
  }
  if (s.bad) return fail(h, TG_BAD_STATE, "non-finite or non-positive state produced by an update");
  return TG_OK;
}

tg_status tg_update_parameters(tg_handle* h, const tg_material* mat, const tg_bc_table* bc) {
  TG_WHOLE_MESH(h)
  if (!h || !mat) return fail(h, TG_INVALID_ARG, "NULL handle or material");
  Params& k = h->prm;
  if (mat->model != k.model || mat->flux_scheme != k.flux || mat->reconstruct_scheme != k.recon ||
      mat->mu_model != k.mu_model)
    return fail(h, TG_NOT_SUPPORTED, "model, flux, reconstruction and viscosity law are fixed at tg_create");
  if (!(mat->gamma > 1.0) || !(mat->gas_const > 0.0)) return fail(h, TG_INVALID_ARG, "gamma must be > 1, gas_const > 0");
  k.gamma = mat->gamma; k.R = mat->gas_const; k.Cp = mat->gamma * mat->gas_const / (mat->gamma - 1.0);
  k.sqrt_gm1 = std::sqrt(mat->gamma - 1.0);
  k.inv_gamma = 1.0 / mat->gamma;
  k.inv_gm1 = 1.0 / (mat->gamma - 1.0);
  k.gp1_gm1 = (mat->gamma + 1.0) / (mat->gamma - 1.0);
  k.prandtl = mat->prandtl; k.mu_ref = mat->mu_ref; k.T0 = mat->T_0; k.Tref = mat->T_ref; k.omega = mat->omega;
  k.ev_alpha = mat->ev_mod_alpha; k.ev_beta = mat->ev_mod_beta; k.tvbM = mat->tvb_minmod_coef;
  k.nd = mat->nd_active; k.visc = mat->visc_active; k.heat = mat->heat_active;
  if (bc && bc->bface_values) {
    HostLayout& L = h->L;
    for (size_t b = 0; b < L.rb_dev.size(); ++b) {
      const int d = L.rb_dev[b];
      if (d < 0) continue;
      for (int q = 0; q < 10; ++q) L.b_val[(size_t)d * 10 + q] = bc->bface_values[b * 10 + q];
    }
    if (!L.b_val.empty())
      TG_CUDA(h, cudaMemcpyAsync(const_cast<double*>(h->mv.b_val), L.b_val.data(), L.b_val.size() * sizeof(double),
                                 cudaMemcpyHostToDevice, h->stream));
  }
  // dt depends on the material; the captured step holds the parameters by value
  clear_dt_next(h);
  drop_graphs(h);
  return sync(h);
}

tg_status tg_output_begin(tg_handle* h, double* prim_out, double* dE_out, int grad_state) {
  TG_WHOLE_MESH(h)
  if (!h || !prim_out) return fail(h, TG_INVALID_ARG, "NULL handle or output buffer");
  if (grad_state != TG_GRAD_LAST_STAGE && grad_state != TG_GRAD_CURRENT)
    return fail(h, TG_INVALID_ARG, "grad_state is TG_GRAD_LAST_STAGE or TG_GRAD_CURRENT");
  if (!host_pinned(prim_out) || (dE_out && !host_pinned(dE_out)))
    return fail(h, TG_INVALID_ARG, "tg_output_begin copies into pinned host memory; tg_get_state takes any buffer");
  const int nv = h->L.nv;
  tg_status st;
  if (!h->snap && (st = dev_alloc(h, 5 * (size_t)nv, &h->snap)) != TG_OK) return st;
  if (dE_out && !h->snap_grad && (st = dev_alloc(h, 15 * (size_t)nv, &h->snap_grad)) != TG_OK) return st;
  if (!h->out_stream) {
    TG_CUDA(h, cudaStreamCreateWithFlags(&h->out_stream, cudaStreamNonBlocking));
    TG_CUDA(h, cudaEventCreateWithFlags(&h->snap_ready, cudaEventDisableTiming));
    TG_CUDA(h, cudaEventCreateWithFlags(&h->out_done, cudaEventDisableTiming));
  }
  // the previous snapshot's copies finish before its buffers are written again
  if (h->out_pending) TG_CUDA(h, cudaStreamWaitEvent(h->stream, h->out_done, 0));
  k_state_out<<<nblk(nv), kBlock, 0, h->stream>>>(nv, h->Pb[0], h->old_of_new, h->snap);
  if (dE_out) {
    // the reference writes the dE of its last compute_gradients: the last stage's input
    // state after a step, the current state after compute_forces of a Navier-Stokes run
    const int last_in = h->ctl.scheme == 1 ? 1 : h->ctl.n_rks - 1;
    refresh_w(h, grad_state == TG_GRAD_CURRENT ? 0 : last_in);
    enqueue_gradient(h, grad_state == TG_GRAD_CURRENT ? 0 : last_in, false, true, h->never);
    k_grad_out<<<nblk(nv), kBlock, 0, h->stream>>>(nv, h->sv.G, h->old_of_new, h->snap_grad, h->sc,
                                                    grad_state == TG_GRAD_LAST_STAGE ? 1 : 0);
  }
  TG_CUDA(h, cudaEventRecord(h->snap_ready, h->stream));
  TG_CUDA(h, cudaStreamWaitEvent(h->out_stream, h->snap_ready, 0));
  TG_CUDA(h, cudaMemcpyAsync(prim_out, h->snap, 5 * (size_t)nv * sizeof(double), cudaMemcpyDeviceToHost, h->out_stream));
  if (dE_out)
    TG_CUDA(h, cudaMemcpyAsync(dE_out, h->snap_grad, 15 * (size_t)nv * sizeof(double), cudaMemcpyDeviceToHost,
                               h->out_stream));
  TG_CUDA(h, cudaEventRecord(h->out_done, h->out_stream));
  h->out_pending = true;
  TG_CUDA(h, cudaGetLastError());
  return TG_OK;
}

tg_status tg_output_wait(tg_handle* h) {
  if (!h) return fail(h, TG_INVALID_ARG, "NULL handle");
  if (!h->out_pending) return TG_OK;
  h->out_pending = false;
  TG_CUDA(h, cudaEventSynchronize(h->out_done));
  return TG_OK;
}

tg_status tg_forces(tg_handle* h, int n_forces, const int* n_tags, const int* tags, double* out) {
  TG_WHOLE_MESH(h)
  if (!h || n_forces < 1 || !n_tags || !tags || !out) return fail(h, TG_INVALID_ARG, "bad force specification");
  std::vector<int> rec4, off;
  const std::string msg = force_faces(h->L, n_forces, n_tags, tags, rec4, off);
  if (!msg.empty()) return fail(h, TG_INVALID_ARG, msg);
  std::vector<int4> rec(rec4.size() / 4);
  for (size_t i = 0; i < rec.size(); ++i) rec[i] = make_int4(rec4[4 * i], rec4[4 * i + 1], rec4[4 * i + 2], rec4[4 * i + 3]);
  tg_status st;
  const int4* drec = nullptr;
  const int* doff = nullptr;
  double* dout = nullptr;
  int4* r = nullptr;
  int* o = nullptr;
  TG_CUDA(h, cudaMalloc((void**)&r, rec.size() * sizeof(int4)));
  TG_CUDA(h, cudaMalloc((void**)&o, off.size() * sizeof(int)));
  TG_CUDA(h, cudaMalloc((void**)&dout, 4 * (size_t)n_forces * sizeof(double)));
  drec = r; doff = o;
  TG_CUDA(h, cudaMemcpyAsync(r, rec.data(), rec.size() * sizeof(int4), cudaMemcpyHostToDevice, h->stream));
  TG_CUDA(h, cudaMemcpyAsync(o, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  // Navier-Stokes forces recompute the gradients of the current state (src/force.cc:123)
  if (h->prm.model == 1) enqueue_gradient(h, 0, false, true, h->never);
  k_forces<<<n_forces, kBlock, 0, h->stream>>>(h->prm, h->mv, view(h, 0), drec, doff, dout);
  std::vector<double> hout(4 * (size_t)n_forces);
  cudaError_t e = cudaMemcpyAsync(hout.data(), dout, hout.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  st = sync(h);
  cudaFree(r); cudaFree(o); cudaFree(dout);
  if (e != cudaSuccess) return fail(h, TG_CUDA_ERROR, cudaGetErrorString(e));
  if (st != TG_OK) return st;
  std::memcpy(out, hout.data(), hout.size() * sizeof(double));
  return TG_OK;
}

tg_status tg_moments_init(tg_handle* h, int n_instances, int extras) {
  TG_WHOLE_MESH(h)
  if (!h) return fail(h, TG_INVALID_ARG, "NULL handle");
  if (n_instances < 1 || extras < 0 || extras > 15) return fail(h, TG_INVALID_ARG, "bad moment layout");
  if (h->mom) { cudaFree(h->mom); h->mom = nullptr; }
  if (h->mom_in) { cudaFree(h->mom_in); h->mom_in = nullptr; }
  h->mom_ninst = n_instances;
  h->mom_extras = extras;
  h->mom_nvar = 5 + ((extras & 1) + ((extras >> 1) & 1) + ((extras >> 2) & 1) + ((extras >> 3) & 1));
  const size_t bytes = (size_t)n_instances * 3 * h->mom_nvar * h->L.nv * sizeof(double);
  TG_CUDA(h, cudaMalloc((void**)&h->mom, bytes));
  TG_CUDA(h, cudaMemsetAsync(h->mom, 0, bytes, h->stream));
  return sync(h);
}

tg_status tg_moments_increment(tg_handle* h, int instance, long k) {
  tg_status st = mom_check(h, instance);
  if (st != TG_OK) return st;
  if (k < 1) return fail(h, TG_INVALID_ARG, "sample index k starts at 1");
  if (h->mom_extras & 8) {
    // vorticity reads dE: the gradients of the initial state before the first
    // step (solve starts with compute_gradients, src/fv.cc:2237), else those of
    // the last stage's input (buffer 2), which the step left in G when its
    // fluxes needed gradients
    Scalars s;
    if ((st = read_scalars(h, &s)) != TG_OK) return st;
    if (s.iter == 0) {
      enqueue_gradient(h, 0, false, true, h->never);
    } else if (!h->grads_needed) {
      refresh_w(h, 2);
      enqueue_gradient(h, 2, false, true, h->never);
    }
  }
  k_moments_increment<<<nblk(h->L.nv), kBlock, 0, h->stream>>>(h->prm, h->L.nv, h->sv.P, h->sv.G, h->mom_extras,
                                                                 h->mom_nvar, (long long)k, mom_array(h, instance, 0),
                                                                 mom_array(h, instance, 1), mom_array(h, instance, 2));
  return sync(h);
}

tg_status tg_moments_get(tg_handle* h, int instance, double* fm, double* sm, double* m2) {
  tg_status st = mom_check(h, instance);
  if (st != TG_OK) return st;
  const size_t nv = h->L.nv, nvar = h->mom_nvar;
  std::vector<double> buf(3 * nvar * nv);
  TG_CUDA(h, cudaMemcpyAsync(buf.data(), mom_array(h, instance, 0), buf.size() * sizeof(double),
                             cudaMemcpyDeviceToHost, h->stream));
  if ((st = sync(h)) != TG_OK) return st;
  double* out[3] = {fm, sm, m2};
  for (int w = 0; w < 3; ++w) {
    if (!out[w]) continue;
    const double* src = buf.data() + (size_t)w * nvar * nv;
    for (size_t i = 0; i < nv; ++i) {
      double* d = out[w] + nvar * (size_t)h->L.old_of_new[i];
      for (size_t c = 0; c < nvar; ++c) d[c] = src[c * nv + i];
    }
  }
  return TG_OK;
}

tg_status tg_moments_export(tg_handle* h, int instance, void* dev_dst) {
  tg_status st = mom_check(h, instance);
  if (st != TG_OK) return st;
  if (!dev_dst) return fail(h, TG_INVALID_ARG, "NULL destination");
  TG_CUDA(h, cudaMemcpyAsync(dev_dst, mom_array(h, instance, 0), 3 * (size_t)h->mom_nvar * h->L.nv * sizeof(double),
                             cudaMemcpyDeviceToDevice, h->stream));
  return sync(h);
}

tg_status tg_moments_merge_device(tg_handle* h, int instance, long n_self, long n_other, const void* dev_group) {
  tg_status st = mom_check(h, instance);
  if (st != TG_OK) return st;
  if (!dev_group || n_self < 0 || n_other < 0 || n_self + n_other < 1) return fail(h, TG_INVALID_ARG, "bad group");
  const size_t n = (size_t)h->mom_nvar * h->L.nv;
  const long n_new = n_self + n_other;
  const double fact1 = (double)n_other / (double)n_new;
  const double fact2 = fact1 * (double)n_self;
  const double* g = (const double*)dev_group;
  k_moments_merge<<<(unsigned)((n + kBlock - 1) / kBlock), kBlock, 0, h->stream>>>(
      n, fact1, fact2, mom_array(h, instance, 0), mom_array(h, instance, 1), mom_array(h, instance, 2), g, g + n,
      g + 2 * n);
  return sync(h);
}

tg_status tg_moments_merge(tg_handle* h, int instance, long n_self, long n_other, const double* fm_o,
                           const double* sm_o, const double* m2_o) {
  tg_status st = mom_check(h, instance);
  if (st != TG_OK) return st;
  if (!fm_o || !sm_o || !m2_o) return fail(h, TG_INVALID_ARG, "NULL group array");
  const size_t nv = h->L.nv, nvar = h->mom_nvar;
  std::vector<double> buf(3 * nvar * nv);
  const double* in[3] = {fm_o, sm_o, m2_o};
  for (int w = 0; w < 3; ++w) {
    double* dst = buf.data() + (size_t)w * nvar * nv;
    for (size_t i = 0; i < nv; ++i) {
      const double* s = in[w] + nvar * (size_t)h->L.old_of_new[i];
      for (size_t c = 0; c < nvar; ++c) dst[c * nv + i] = s[c];
    }
  }
  if (!h->mom_in) TG_CUDA(h, cudaMalloc((void**)&h->mom_in, buf.size() * sizeof(double)));
  TG_CUDA(h, cudaMemcpyAsync(h->mom_in, buf.data(), buf.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  return tg_moments_merge_device(h, instance, n_self, n_other, h->mom_in);
}

tg_status tg_moments_finalize(tg_handle* h, int instance, long n) {
  tg_status st = mom_check(h, instance);
  if (st != TG_OK) return st;
  if (n < 2) return fail(h, TG_INVALID_ARG, "moments need at least two samples (src/parameter.cc:804-805)");
  const size_t m = (size_t)h->mom_nvar * h->L.nv;
  k_moments_scale<<<(unsigned)((m + kBlock - 1) / kBlock), kBlock, 0, h->stream>>>(
      m, 1.0 / ((double)n - 1.0), 1.0 / (double)n, mom_array(h, instance, 1), mom_array(h, instance, 2));
  return sync(h);
}

tg_status tg_global(tg_handle* h, double* ke, double* ent) {
  TG_WHOLE_MESH(h)
  if (!h) return fail(h, TG_INVALID_ARG, "NULL handle");
  k_global<<<h->nblocks_v, kBlock, 0, h->stream>>>(h->prm, h->mv, view(h, 0));
  std::vector<double> part(4 * (size_t)h->nblocks_v);
  TG_CUDA(h, cudaMemcpyAsync(part.data(), h->sv.part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  tg_status st = sync(h);
  if (st != TG_OK) return st;
  double a = 0.0, b = 0.0;
  for (int i = 0; i < h->nblocks_v; ++i) { a += part[4 * (size_t)i]; b += part[4 * (size_t)i + 1]; }
  if (ke) *ke = a;
  if (ent) *ent = b;
  return TG_OK;
}

tg_status tg_stream(tg_handle* h, void** out) {
  if (!h || !out) return fail(h, TG_INVALID_ARG, "NULL argument");
  *out = (void*)h->stream;
  return TG_OK;
}

tg_status tg_time_phase(tg_handle* h, int phase, int reps, double* ms) {
  TG_WHOLE_MESH(h)
  if (!h || !ms || reps <= 0 || phase < 0 || phase > 4) return fail(h, TG_INVALID_ARG, "bad argument");
  if (phase == TG_PHASE_STEP) {
    tg_status st = capture_step_graph(h);
    if (st != TG_OK) return st;
  }
  cudaEvent_t a, b;
  TG_CUDA(h, cudaEventCreate(&a));
  TG_CUDA(h, cudaEventCreate(&b));
  enqueue_phase(h, phase);
  TG_CUDA(h, cudaEventRecord(a, h->stream));
  for (int i = 0; i < reps; ++i) enqueue_phase(h, phase);
  TG_CUDA(h, cudaEventRecord(b, h->stream));
  tg_status st = sync(h);
  float t = 0.0f;
  if (st == TG_OK) {
    cudaError_t e = cudaEventElapsedTime(&t, a, b);
    if (e != cudaSuccess) st = fail(h, TG_CUDA_ERROR, cudaGetErrorString(e));
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = (double)t / reps;
  return st;
}

tg_status tg_query(tg_handle* h, int key, double* out) {
  if (!h || !out) return fail(h, TG_INVALID_ARG, "NULL argument");
  switch (key) {
    case TG_Q_N_VERTEX: *out = h->mv.nv; break;
    case TG_Q_N_EDGE: *out = h->mv.ne; break;
    case TG_Q_N_BFACE: *out = h->mv.nb; break;
    case TG_Q_KERNELS_PER_STEP: *out = h->kernels_per_step; break;
    case TG_Q_DEVICE_BYTES: *out = (double)h->device_bytes; break;
    case TG_Q_KERNELS_PER_PHASE: *out = h->kernels_per_flux; break;
    case TG_Q_N_TILES: *out = h->L.ntiles; break;
    case TG_Q_RESIDUAL_NORM0: {
      Scalars s;
      const tg_status st = read_scalars(h, &s);
      if (st != TG_OK) return st;
      *out = s.rtotal0;
      break;
    }
    default: return fail(h, TG_INVALID_ARG, "unknown query key");
  }
  return TG_OK;
}

// ---- domain decomposition

tg_status tg_part_plan(const tg_mesh* mesh, const tg_bc_table* bc, int n_parts, int part, int* out4, int* local,
                       int* send_counts, int* recv_counts, int* send_idx, int* recv_idx) {
  if (!mesh || !out4) return fail(nullptr, TG_INVALID_ARG, "NULL argument");
  HostLayout G;
  std::string msg = build_layout(*mesh, bc, false, G);
  PartPlan P;
  if (msg.empty()) msg = plan_partition(G, n_parts, part, P);
  if (!msg.empty()) return fail(nullptr, TG_INVALID_ARG, msg);
  out4[0] = P.n_owned;
  out4[1] = (int)P.local.size() - P.n_owned;
  out4[2] = (int)P.send_idx.size();
  out4[3] = (int)P.recv_idx.size();
  if (local)
    for (size_t i = 0; i < P.local.size(); ++i) local[i] = G.old_of_new[P.local[i]];
  for (int q = 0; q < n_parts; ++q) {
    if (send_counts) send_counts[q] = P.send_off[q + 1] - P.send_off[q];
    if (recv_counts) recv_counts[q] = P.recv_off[q + 1] - P.recv_off[q];
  }
  if (send_idx) std::copy(P.send_idx.begin(), P.send_idx.end(), send_idx);
  if (recv_idx) std::copy(P.recv_idx.begin(), P.recv_idx.end(), recv_idx);
  return TG_OK;
}

tg_status tg_part_create(const tg_mesh* mesh, const tg_material* mat, const tg_bc_table* bc, const tg_options* opt,
                         int n_parts, int part, tg_handle** out) {
  if (n_parts < 1 || part < 0 || part >= n_parts) return fail(nullptr, TG_INVALID_ARG, "partition index out of range");
  return create_handle(mesh, mat, bc, opt, n_parts, part, out);
}

}  // extern "C"

namespace {

tg_status part_check(tg_handle* h) {
  if (!h) return fail(h, TG_INVALID_ARG, "NULL handle");
  if (h->part.n_parts == 0) return fail(h, TG_INVALID_ARG, "not a partition handle (tg_part_create)");
  return TG_OK;
}

// buffers stage r reads and writes (as enqueue_step rotates them)
void stage_buffers(const tg_handle* h, int r, int* bin, int* bout) {
  const int rk4_in[4] = {0, 1, 2, 1}, rk4_out[4] = {1, 2, 1, 0};
  *bin = h->ctl.scheme == 1 ? rk4_in[r] : r;
  *bout = h->ctl.scheme == 1 ? rk4_out[r] : (r + 1) % 3;
}

tg_status launched(tg_handle* h) {
  TG_CUDA(h, cudaGetLastError());
  return TG_OK;
}

}  // namespace

extern "C" {

tg_status tg_part_info(tg_handle* h, int* out8, int* send_counts, int* recv_counts) {
  tg_status st = part_check(h);
  if (st != TG_OK) return st;
  if (!out8) return fail(h, TG_INVALID_ARG, "NULL argument");
  const auto& P = h->part;
  out8[0] = P.n_parts; out8[1] = P.part; out8[2] = P.n_owned; out8[3] = h->L.nv - P.n_owned;
  out8[4] = P.n_send; out8[5] = P.n_recv; out8[6] = h->L.ntiles; out8[7] = P.n_frontier;
  for (int q = 0; q < P.n_parts; ++q) {
    if (send_counts) send_counts[q] = P.send_off[q + 1] - P.send_off[q];
    if (recv_counts) recv_counts[q] = P.recv_off[q + 1] - P.recv_off[q];
  }
  return TG_OK;
}

tg_status tg_part_prime(tg_handle* h) {
  tg_status st = part_check(h);
  if (st != TG_OK) return st;
  if (h->prm.fuse_dt) {
    grad_kernel(true, false)<<<h->L.ntiles, kTileThreads, h->smem_grad1, h->stream>>>(
        h->prm, h->mv, h->tv, view(h, 0), h->sc, h->L.lmax, h->L.emax, h->never, 0);
    k_part_primed<<<1, 1, 0, h->stream>>>(h->sc);
  }
  h->cold = false;
  return launched(h);
}

tg_status tg_part_begin(tg_handle* h) {
  tg_status st = part_check(h);
  if (st != TG_OK) return st;
  if (h->cold) return fail(h, TG_INVALID_ARG, "tg_part_prime and the scalar exchange come first after a new state");
  k_step_begin<<<1, 1, 0, h->stream>>>(h->ctl, h->sc, h->done, 1);
  if (h->ctl.time_step > 0.0) k_store_old<<<nblk(h->mv.nv), kBlock, 0, h->stream>>>(h->prm, h->mv, view(h, 0), h->done);
  return launched(h);
}

}  // extern "C"

namespace {

// The tiles a stage call covers: all, the frontier [0, n_frontier) or the interior.
tg_status part_tiles(tg_handle* h, int which, int* base, int* count) {
  const int nf = h->part.n_frontier, nt = h->L.ntiles;
  switch (which) {
    case TG_TILES_ALL: *base = 0; *count = nt; return TG_OK;
    case TG_TILES_FRONTIER: *base = 0; *count = nf; return TG_OK;
    case TG_TILES_INTERIOR: *base = nf; *count = nt - nf; return TG_OK;
    default: return fail(h, TG_INVALID_ARG, "unknown tile set");
  }
}

}  // namespace

extern "C" {

tg_status tg_part_gradients(tg_handle* h, int r, int which) {
  tg_status st = part_check(h);
  if (st != TG_OK) return st;
  if (r < 0 || r >= h->ctl.n_rks) return fail(h, TG_INVALID_ARG, "stage out of range");
  int bin, bout, base, count;
  if ((st = part_tiles(h, which, &base, &count)) != TG_OK) return st;
  stage_buffers(h, r, &bin, &bout);
  enqueue_gradient(h, bin, false, h->grads_needed, h->done, base, count);
  return launched(h);
}

tg_status tg_part_flux(tg_handle* h, int r, int which) {
  tg_status st = part_check(h);
  if (st != TG_OK) return st;
  if (r < 0 || r >= h->ctl.n_rks) return fail(h, TG_INVALID_ARG, "stage out of range");
  int bin, bout, base, count;
  if ((st = part_tiles(h, which, &base, &count)) != TG_OK) return st;
  stage_buffers(h, r, &bin, &bout);
  const bool last = r == h->ctl.n_rks - 1;
  // boundary-face sides depend only on their own vertex's state: the faces are formed with
  // the interior (or all) tiles, and the frontier tiles, launched after, gather them too
  if (which != TG_TILES_FRONTIER) enqueue_boundary(h, bin, h->done);
  enqueue_tile_flux(h, bin, MODE_UPDATE, r, last, bout, h->done, base, count);
  if (which != TG_TILES_INTERIOR) {
    h->part.cur = bout;
    if (last) h->part.norms_pending = true;
  }
  return launched(h);
}

tg_status tg_part_pack(tg_handle* h, int field, void* dev_send) {
  tg_status st = part_check(h);
  if (st != TG_OK) return st;
  if (field != TG_HALO_STATE && field != TG_HALO_GRAD) return fail(h, TG_INVALID_ARG, "unknown halo field");
  const int n = h->part.n_send, nv = h->L.nv;
  if (n == 0) return TG_OK;
  if (!dev_send) return fail(h, TG_INVALID_ARG, "NULL send buffer");
  const double* A = field == TG_HALO_STATE ? h->Pb[h->part.cur] : h->sv.G;
  const double* B = field == TG_HALO_STATE ? h->Wb[h->part.cur] : h->sv.G + 4 * (size_t)nv;
  k_halo_pack<<<nblk(8 * n), kBlock, 0, h->stream>>>(n, h->part.send_idx, nv, A, B, (double*)dev_send);
  return launched(h);
}

tg_status tg_part_unpack(tg_handle* h, int field, const void* dev_recv) {
  tg_status st = part_check(h);
  if (st != TG_OK) return st;
  if (field != TG_HALO_STATE && field != TG_HALO_GRAD) return fail(h, TG_INVALID_ARG, "unknown halo field");
  const int n = h->part.n_recv, nv = h->L.nv;
  if (n == 0) return TG_OK;
  if (!dev_recv) return fail(h, TG_INVALID_ARG, "NULL receive buffer");
  double* A = field == TG_HALO_STATE ? h->Pb[h->part.cur] : h->sv.G;
  double* B = field == TG_HALO_STATE ? h->Wb[h->part.cur] : h->sv.G + 4 * (size_t)nv;
  k_halo_unpack<<<nblk(8 * n), kBlock, 0, h->stream>>>(n, h->part.recv_idx, nv, A, B, (const double*)dev_recv);
  return launched(h);
}

tg_status tg_part_export(tg_handle* h, void* dev_out) {
  tg_status st = part_check(h);
  if (st != TG_OK) return st;
  if (!dev_out) return fail(h, TG_INVALID_ARG, "NULL buffer");
  k_part_export<<<1, 1, 0, h->stream>>>(h->sc, (unsigned long long*)dev_out);
  return launched(h);
}

tg_status tg_part_import(tg_handle* h, const void* dev_all) {
  tg_status st = part_check(h);
  if (st != TG_OK) return st;
  if (!dev_all) return fail(h, TG_INVALID_ARG, "NULL buffer");
  k_part_import<<<1, 1, 0, h->stream>>>(h->sc, (const unsigned long long*)dev_all, h->part.n_parts, h->n_caller,
                                        h->part.norms_pending ? 1 : 0);
  h->part.norms_pending = false;
  return launched(h);
}

tg_status tg_part_scalars(tg_handle* h, double* info4) {
  tg_status st = part_check(h);
  if (st != TG_OK) return st;
  Scalars s;
  if ((st = read_scalars(h, &s)) != TG_OK) return st;
  if (info4) { info4[0] = s.elapsed; info4[1] = s.dt_global; info4[2] = s.rtotal; info4[3] = (double)s.iter; }
  if (s.bad) return fail(h, TG_BAD_STATE, "non-finite or non-positive state produced by an update");
  return TG_OK;
}

}  // extern "C"
