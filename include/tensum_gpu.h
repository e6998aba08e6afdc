/*
 * tensum_gpu.h -- C ABI of the B200 residual/update path for TENSUM's 2D
 * vertex-centred median-dual finite-volume solver.
 *
 * Drop-in boundary.  In the reference the hot path is reached through private
 * members of FiniteVolume (src/fv.h:351-403) called from FiniteVolume::solve
 * (src/fv.cc:2273-2305), operating on the member arrays primitive,
 * conserved_old, entropy_var, residual, dE, dE_cell, dt (src/fv.h:137-164) and
 * on the public Grid data (src/grid.h:141-229).  Each entry point below
 * replaces one of those calls; the caller keeps the reference's parameter
 * reader, part-file reader, Grid::preproc and writers unchanged and hands the
 * resulting arrays across this ABI.
 *
 * Conventions
 *  - Plain C types only; every pointer is a HOST pointer unless the name ends
 *    in _dev.  Arrays use the reference's local vertex/cell/face numbering.
 *  - Every call returns tg_status; nothing throws across the ABI.  After a
 *    failure tg_last_error(h) returns a message (thread-local when h is NULL).
 *  - One host thread per handle.  Calls are ordered on the handle's CUDA
 *    stream and return after the work is complete unless documented otherwise.
 *  - The device path has no CPU fallback: without a usable CUDA device
 *    tg_create returns TG_NO_DEVICE.
 */
#ifndef TENSUM_GPU_H
#define TENSUM_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define TG_ABI_VERSION 4

typedef enum {
  TG_OK = 0,
  TG_BAD_STATE = 1,     /* non-finite value or p <= 0 / rho <= 0 seen in an update   */
  TG_TIMEOUT = 2,       /* a bounded device wait ran out                            */
  TG_CUDA_ERROR = 3,    /* a CUDA runtime call failed                               */
  TG_INVALID_ARG = 4,   /* malformed mesh / option / size                           */
  TG_NOT_SUPPORTED = 5, /* option the device path does not implement               */
  TG_NO_DEVICE = 6      /* no CUDA device visible                                   */
} tg_status;

/* Material::FluxScheme, src/material.h:78-91 (same order). */
typedef enum {
  TG_FLUX_KEPES_TECNO_ROE = 0,
  TG_FLUX_KEPES_TECNO_RUSANOV = 1,
  TG_FLUX_KEPEC = 2,
  TG_FLUX_ROE_EC = 3,
  TG_FLUX_KEP = 4,
  TG_FLUX_AVG = 5
} tg_flux_scheme;

/* Material::ReconstructScheme, src/material.h:97-106 (same order). */
typedef enum {
  TG_RECON_FIRST = 0,
  TG_RECON_SECOND = 1,
  TG_RECON_SECOND_MUSCL = 2,
  TG_RECON_VAN_ALBADA = 3,
  TG_RECON_TVD_MINMOD = 4,
  TG_RECON_TVB_MINMOD = 5,
  TG_RECON_ENO2 = 6
} tg_reconstruct_scheme;

/* Material::MuModel, src/material.h:92-95. */
typedef enum { TG_MU_CONSTANT = 0, TG_MU_SUTHERLAND = 1, TG_MU_POWER = 2 } tg_mu_model;

/* BC::BCType, src/bc.h:16-25 (same order). */
typedef enum {
  TG_BC_NONE = 0,
  TG_BC_SLIP = 1,
  TG_BC_NOSLIP = 2,
  TG_BC_FARFIELD = 3,
  TG_BC_INLET = 4,
  TG_BC_OUTLET = 5,
  TG_BC_PRESSURE = 6,
  TG_BC_PERIODIC = 7
} tg_bc_kind;

/*
 * Mesh after Grid::preproc (src/grid_preproc.cc:1147-1194), one partition,
 * median or Voronoi dual, planar or axisymmetric.  Field-by-field the members of Grid:
 *   coords        vertex[i].coord.{x,y}                      2*n_vertex
 *   dcarea/mcarea dual / median areas, periodic-summed        n_vertex
 *   cell_vertex   cell[c].vertex[0..2]                        3*n_cell
 *   cell_normal   cell[c].normal[k].{x,y} (P1 normals)        6*n_cell
 *   cell_area     cell[c].area                                n_cell
 *   face_*        face[f]: vertex[0..1], type (-1 interior, else boundary tag),
 *                 normal.{x,y} (dual-face normal), lcell, rcell (-1 if none).
 *                 Boundary faces come first, face[i] <-> bface[i].
 *   bface_*       bface[b]: vertex[0..1], type, normal.{x,y} (outward),
 *                 lcell, periodic flag.
 *   periodic_*    periodic_lists[i].P_ij as CSR (offsets n_periodic+1).
 *   *_radius      vertex[i].radius, face[f].radius, cell[c].radius of an
 *                 axisymmetric run (-axi, src/grid_preproc.cc:750-777: the x of
 *                 the vertex, face centre and cell centre); all three NULL for
 *                 a planar mesh (radius 1 everywhere).
 */
typedef struct {
  int n_vertex;
  const double* coords;
  const double* dcarea;
  const double* mcarea;
  int n_cell;
  const int* cell_vertex;
  const double* cell_normal;
  const double* cell_area;
  int n_face;
  const int* face_vertex;
  const int* face_type;
  const double* face_normal;
  const int* face_lcell;
  const int* face_rcell;
  int n_bface;
  const int* bface_vertex;
  const int* bface_type;
  const double* bface_normal;
  const int* bface_lcell;
  const unsigned char* bface_periodic;
  int n_periodic;
  const int* periodic_offsets;
  const int* periodic_members;
  const double* vertex_radius;
  const double* face_radius;
  const double* cell_radius;
} tg_mesh;

/* class Material, src/material.h:54-420 (data members). */
typedef struct {
  double gamma;
  double gas_const;
  double prandtl;
  double mu_ref;
  double T_0;
  double T_ref;
  double omega;
  double ev_mod_alpha;
  double ev_mod_beta;
  double tvb_minmod_coef;
  int model;               /* 0 = euler, 1 = ns (Material::FlowModel) */
  int flux_scheme;         /* tg_flux_scheme */
  int mu_model;            /* tg_mu_model */
  int reconstruct_scheme;  /* tg_reconstruct_scheme */
  int nd_active;
  int visc_active;
  int heat_active;
} tg_material;

/*
 * Boundary conditions.  The reference evaluates fparser expressions of (x,y,t)
 * per boundary vertex inside BoundaryCondition::apply (src/bc.h:568-654); for
 * SSP-RK3 the time argument is never advanced, so the caller evaluates them
 * once and passes the values per boundary-face vertex:
 *   bface_values[(2*b + k)*5 + {0..4}] = (T, u, v, w, p) at bface[b].vertex[k].
 * Components a kind does not use are ignored; bface_values may be NULL when
 * every kind is periodic/slip/outlet.
 */
typedef struct {
  int n_types;
  const int* type_tag;             /* boundary tag (face type)                   */
  const int* kind;                 /* tg_bc_kind per tag                         */
  const unsigned char* adiabatic;  /* BoundaryCondition::adiabatic per tag        */
  const double* bface_values;      /* n_bface*2*5 or NULL                         */
} tg_bc_table;

typedef enum { TG_TIME_SSPRK3 = 0, TG_TIME_RK4 = 1, TG_TIME_HEUNS = 2 } tg_time_scheme;
typedef enum { TG_STEADY = 0, TG_UNSTEADY = 1 } tg_time_mode;

/* Parameter members of the numeric/output sections, src/parameter.h. */
typedef struct {
  int time_scheme;      /* tg_time_scheme                                         */
  int time_mode;        /* tg_time_mode                                           */
  double time_step;     /* > 0: fixed global step (src/fv.cc:1503-1509)           */
  double cfl;
  double final_time;
  int n_time_stamps;    /* unsteady output instances: t_i = i*final_time/n        */
  long max_iter;
  double min_residue;
  int bad_state_check;  /* nonzero: flag non-finite / p<=0 / rho<=0 in updates  */
  int liou_fix;         /* numeric liou_fix: Liou's carbuncle switch for kepes_tecno_roe */
  int bc_strong;        /* numeric bc_scheme strong (1) or weak (0)                */
} tg_options;

typedef struct tg_handle tg_handle;

/* ---- lifetime ---------------------------------------------------------- */

/* Replaces FiniteVolume::initialize (src/fv.cc:25-197) for the hot path:
 * validates the mesh, builds the device layout, allocates all device memory. */
tg_status tg_create(const tg_mesh* mesh, const tg_material* mat, const tg_bc_table* bc,
                    const tg_options* opt, tg_handle** out);
tg_status tg_destroy(tg_handle* h);
const char* tg_last_error(const tg_handle* h);
int tg_abi_version(void);

/* ---- state ------------------------------------------------------------- */

/* primitive[] <- prim_aos (T,p,u,v,w per vertex: the PrimVar layout of src/primvar.h:17-18),
 * then entropy_var = prim2ent(primitive) (src/fv.cc:392-393).  Resets time to t0. */
tg_status tg_set_state(tg_handle* h, const double* prim_aos, int n_vertex, double t0);
/* Queue a new state (PrimVar records in the caller's order, from PINNED host
 * memory, starting at time t0) and return at once: its copy to the device runs
 * on a side stream while the handle keeps working, and the next tg_step or
 * tg_advance takes it in before its first step, exactly as tg_set_state would
 * (at most two states queued; they are taken in order).  The buffer must stay
 * unchanged until that tg_step / tg_advance has returned.  A refused state
 * (T <= 0 or p <= 0, src/fv.cc:388-389) is reported by that call as
 * TG_INVALID_ARG, after its steps ran on the previous state.  tg_set_state
 * drops queued states.  With tg_output_begin this lets a caller stream states
 * in and results out while the device steps. */
tg_status tg_set_state_async(tg_handle* h, const double* prim_aos, int n_vertex, double t0);

/* prim_aos <- primitive[] (periodic copies receive their set's value). */
tg_status tg_get_state(tg_handle* h, double* prim_aos, int n_vertex);

/* ---- hot path, one call per reference member function ----------------- */

/* store_conserved_old (src/fv.cc:1626-1630). */
tg_status tg_store_conserved_old(tg_handle* h);
/* compute_dt (src/fv.cc:1499-1621): local dt, periodic sum, global min and the
 * unsteady clamp to the next output time.  dt_out (n_vertex) may be NULL. */
tg_status tg_compute_dt(tg_handle* h, double* dt_global_out, double* dt_out);
/* compute_gradients (src/fv.cc:699-1059): dE_out is n_vertex*5*3 in the
 * reference layout dE[v][var][xyz] (var order V1,V2,V3,V4,V5; z = 0). May be NULL. */
tg_status tg_gradients(tg_handle* h, double* dE_out);
/* compute_residual (src/fv.cc:1467-1494): gradients + inviscid + viscous +
 * periodic sum.  res_out is n_vertex*5 in Flux layout (mass, mx, my, mz, energy). */
tg_status tg_residual(tg_handle* h, double* res_out);
/* update_solution(r) for SSP-RK3 (src/fv.cc:1635-1658). */
tg_status tg_update(tg_handle* h, int r);
/* compute_residual_norm (src/fv.cc:1801-1879) on the current residual.
 * out[0..5] = mass, mx, my, energy norms, total (normalised), total0. */
tg_status tg_residual_norm(tg_handle* h, long iter, double* out6);

/* Tail of one solve-loop iteration (src/fv.cc:2307-2343): iteration count +1,
 * elapsed_time += dt_global, advance the output-time counter when reached.
 * Used with the single-phase calls above; tg_step does it itself.
 * info4 as for tg_step (may be NULL). */
tg_status tg_end_step(tg_handle* h, double* info4);

/* One or more complete time steps of FiniteVolume::solve's loop
 * (src/fv.cc:2273-2316): store_conserved_old, compute_dt, n_rks x
 * (compute_residual, [norm at last stage], update_solution), t += dt.
 * Steps after final_time is reached are no-ops.  info (may be NULL) receives
 * {elapsed_time, dt_global, residual_norm_total, iterations_done}. */
tg_status tg_step(tg_handle* h, int n_steps, double* info4);

/* Global kinetic energy and entropy integrals, compute_global (src/fv.cc:2175-2225). */
tg_status tg_global(tg_handle* h, double* ke_out, double* entropy_out);

/* New material constants and boundary values for the same mesh, e.g. per Monte
 * Carlo sample whose inflow or viscosity is uncertain (the reference re-reads
 * them per sample through its expressions).  The model, flux, reconstruction,
 * viscosity law and the tag -> boundary-kind mapping stay those of tg_create;
 * bc may be NULL (values kept).  The state is untouched. */
tg_status tg_update_parameters(tg_handle* h, const tg_material* mat, const tg_bc_table* bc);

/* Output at an output time (the writers of src/writer.cc:129-409,
 * src/output_skin_friction.cc, src/output_heatflux.cc read primitive and dE):
 * tg_output_begin snapshots the current state, as PrimVar records in the
 * caller's vertex order, and optionally the entropy-variable gradients as the
 * reference's dE records (n_vertex x 5 variables x (x, y, z)), on the device,
 * then copies them into the caller's PINNED buffers on a side stream and
 * returns; steps enqueued afterwards overlap the copy.  tg_output_wait blocks
 * until the copy is complete.  grad_state selects which gradients the
 * reference would hold: TG_GRAD_LAST_STAGE those of the last stage's input
 * state (after a step; zero before any step), TG_GRAD_CURRENT those of the
 * current state (after compute_forces of a Navier-Stokes run). */
enum { TG_GRAD_LAST_STAGE = 0, TG_GRAD_CURRENT = 1 };
tg_status tg_output_begin(tg_handle* h, double* prim_aos, double* dE_aos, int grad_state);
tg_status tg_output_wait(tg_handle* h);

/* compute_forces (src/force.cc:116-219) on the current state: for each force
 * f (its face tags are tags[sum n_tags[<f] .. +n_tags[f]), the integrals over
 * its boundary faces of the pressure force and, for Navier-Stokes, the viscous
 * stress.  out[4f..4f+3] = inviscid x, y, viscous x, y.  Like the reference
 * it applies the boundary condition of bface[f] (f the force index) on every
 * face of force f. */
tg_status tg_forces(tg_handle* h, int n_forces, const int* n_tags, const int* tags, double* out4);

/* Steps, as tg_step, until output time `instance` has been reached (the
 * unsteady counter of src/fv.cc:2317-2336 exceeds it), the run is over, or
 * max_steps steps have been issued (a step past the stop is a no-op).
 * info5 (may be NULL): tg_step's four values, then the output-time counter. */
tg_status tg_advance(tg_handle* h, int instance, long max_steps, double* info5);

/* ---- Monte Carlo moments ---------------------------------------------- */
/* The per-group online statistics of increment_moments (src/fv.cc:595-694) and
 * their reduction over groups, reduce_moments (src/reduce_moments.cc:14-221).
 * Per output instance the handle keeps fm (running mean), sm (sum of squares)
 * and m2 (sum of squared deviations), each n_vertex records of nvar doubles:
 * PrimVar (T, p, u, v, w), then density, mach, entropy and vorticity for the
 * bits 1, 2, 4, 8 of `extras` (the output section's write_variables), in the
 * order reduce_moments packs them.  Host arrays are in the caller's vertex
 * order; device group blocks (tg_moments_export) are three [nvar][n_vertex]
 * arrays fm, sm, m2 in the handle's internal vertex order. */
tg_status tg_moments_init(tg_handle* h, int n_instances, int extras);
/* increment_moments at output `instance` for the k-th sample of the group
 * (k = 1 starts the group).  Vorticity uses the gradients of the state's
 * last residual evaluation, or of the state itself before its first step. */
tg_status tg_moments_increment(tg_handle* h, int instance, long k);
/* Raw group moments of one instance to host arrays (any may be NULL). */
tg_status tg_moments_get(tg_handle* h, int instance, double* fm, double* sm, double* m2);
/* The group block of one instance into caller device memory (3*nvar*n_vertex doubles). */
tg_status tg_moments_export(tg_handle* h, int instance, void* dev_dst);
/* Merge another group (n_other samples) into this one (n_self samples), the
 * per-group update of reduce_moments; from host arrays or a device block. */
tg_status tg_moments_merge(tg_handle* h, int instance, long n_self, long n_other, const double* fm_other,
                           const double* sm_other, const double* m2_other);
tg_status tg_moments_merge_device(tg_handle* h, int instance, long n_self, long n_other, const void* dev_group);
/* reduce_moments' final scaling for n samples in all: m2 /= (n-1), sm /= n. */
tg_status tg_moments_finalize(tg_handle* h, int instance, long n);

/* ---- measurement (no counterpart in the reference, whose Timer class,
 *      src/timer.h:8-72, wraps MPI_Wtime around each phase) -------------- */

/* The CUDA stream (cudaStream_t) every call of this handle is ordered on, so a
 * caller can bracket calls with its own CUDA events. */
tg_status tg_stream(tg_handle* h, void** stream_out);

/* ---- measurement hooks: extensions with no counterpart in the reference ----
 * tg_time_phase, tg_query and tg_batch_time_steps exist for benchmarks and
 * tests (device time of one phase, layout facts); a drop-in caller does not
 * need them. */
typedef enum {
  TG_PHASE_GRADIENT = 0,   /* compute_gradients                                   */
  TG_PHASE_FLUX = 1,       /* inviscid + viscous fluxes and residual assembly     */
  TG_PHASE_UPDATE = 2,     /* update_solution (changes the state)                 */
  TG_PHASE_DT = 3,         /* compute_dt                                          */
  TG_PHASE_STEP = 4        /* one full time step (graph replay)                   */
} tg_phase;

/* Average device time of one phase over `reps` back-to-back launches, measured
 * with CUDA events on the handle's stream after one untimed launch. */
tg_status tg_time_phase(tg_handle* h, int phase, int reps, double* ms_per_launch);

typedef enum {
  TG_Q_N_VERTEX = 0,
  TG_Q_N_EDGE = 1,
  TG_Q_N_BFACE = 2,
  TG_Q_KERNELS_PER_STEP = 3,   /* kernel launches in one tg_step step        */
  TG_Q_DEVICE_BYTES = 4,       /* device memory owned by the handle          */
  TG_Q_KERNELS_PER_PHASE = 5,  /* launches of one TG_PHASE_FLUX call         */
  TG_Q_N_TILES = 6,            /* vertex tiles (CTAs of one tiled pass)      */
  TG_Q_RESIDUAL_NORM0 = 7      /* residual_norm_total0, the normaliser of the */
                               /* relative norm (restart files, src/writer.cc) */
} tg_query_key;
tg_status tg_query(tg_handle* h, int key, double* out);

/* ---- domain decomposition of one mesh -----------------------------------
 * Replaces the reference's MPI partitions of one mesh (read_part_mesh_file.cc,
 * the shared-vertex residual and gradient sums of src/reduce_residual.cc:14-104
 * and src/fv.cc:827-1030, the dt minimum of src/fv.cc:1602 and the norm sum of
 * src/reduce_res_norm.cc:25).  The vertices, in the solver's Hilbert order,
 * are cut into n_parts contiguous ranges; a partition owns one range and holds as
 * ghosts every vertex its owned vertices' gather lists reach.  Each vertex is
 * computed only by its owner, in the one-partition order, so any partition count
 * gives the one-partition result bit for bit.  Inviscid runs with weak boundary
 * conditions (no strong conditions, no Liou fix).  One process per GPU, each with
 * its partition handle, is the intended use; the exchange is the caller's (NCCL
 * all-to-all and all-gather over NVLink, or device copies in one process).
 *
 * A step, every call enqueued on the handle's stream (tg_stream), no host wait:
 *   tg_part_begin
 *   for each stage r:  tg_part_gradients(r, TG_TILES_ALL), exchange TG_HALO_GRAD,
 *                      tg_part_flux(r, TG_TILES_ALL),      exchange TG_HALO_STATE
 *   tg_part_export, all-gather of the 5-word records in partition order, tg_part_import
 * The tiles are ordered frontier first (tiles that read a ghost), interior after; the
 * interior tiles need no ghost, so each exchange can overlap them:
 *   gradients(r, INTERIOR) | finish STATE | gradients(r, FRONTIER) | start GRAD |
 *   flux(r, INTERIOR) | finish GRAD | flux(r, FRONTIER) | start STATE
 * (without gradients: flux(r, INTERIOR) | finish STATE | flux(r, FRONTIER) | start STATE).
 * An exchange of a field: tg_part_pack into the send buffer (8 doubles per
 * vertex, peers in ascending order, send_counts[q] vertices for peer q), the
 * all-to-all, tg_part_unpack from the receive buffer (recv_counts[q] vertices
 * from peer q, peers ascending).  After tg_set_state (the whole mesh's records):
 * tg_part_prime, then the scalar exchange, before the first tg_part_begin. */
enum { TG_HALO_STATE = 0, TG_HALO_GRAD = 1 };
enum { TG_TILES_ALL = 0, TG_TILES_FRONTIER = 1, TG_TILES_INTERIOR = 2 };

/* Host only (no device): the plan of partition `part`.  out4 = {n_owned, n_ghost,
 * n_send, n_recv}; the optional arrays receive the caller indices of the
 * partition's vertices (owned first, n_owned + n_ghost), the per-peer counts
 * (n_parts each) and the local positions of the send / receive entries. */
tg_status tg_part_plan(const tg_mesh* mesh, const tg_bc_table* bc, int n_parts, int part, int* out4, int* local,
                       int* send_counts, int* recv_counts, int* send_idx, int* recv_idx);
tg_status tg_part_create(const tg_mesh* mesh, const tg_material* mat, const tg_bc_table* bc, const tg_options* opt,
                         int n_parts, int part, tg_handle** out);
/* out8 = {n_parts, part, n_owned, n_ghost, n_send, n_recv, n_tiles, n_frontier_tiles};
 * counts per peer. */
tg_status tg_part_info(tg_handle* h, int* out8, int* send_counts, int* recv_counts);
/* Local dt and U_old of the owned vertices of a new state (the first-stage dt pass). */
tg_status tg_part_prime(tg_handle* h);
tg_status tg_part_begin(tg_handle* h);
/* tiles: TG_TILES_ALL, or TG_TILES_FRONTIER and TG_TILES_INTERIOR in either order. */
tg_status tg_part_gradients(tg_handle* h, int stage, int tiles);
/* Boundary and edge fluxes and the stage update; the last stage also forms the
 * next step's local dt and U_old and this partition's residual-norm sums.  tiles:
 * TG_TILES_ALL, or TG_TILES_INTERIOR followed by TG_TILES_FRONTIER. */
tg_status tg_part_flux(tg_handle* h, int stage, int tiles);
tg_status tg_part_pack(tg_handle* h, int field, void* dev_send);
tg_status tg_part_unpack(tg_handle* h, int field, const void* dev_recv);
/* 5 x 8 bytes: the dt minimum (bits) and the four residual-norm sums. */
tg_status tg_part_export(tg_handle* h, void* dev_out);
/* n_parts x 5 x 8 bytes in partition order: every partition forms the same dt and norms. */
tg_status tg_part_import(tg_handle* h, const void* dev_all);
/* Waits for the stream; info4 = {elapsed, dt, relative residual, iteration}. */
tg_status tg_part_scalars(tg_handle* h, double* info4);

/* ---- batched FP32 ensembles (no counterpart in the reference, which runs
 *      one sample after another per MC group, src/fv.cc:2440-2456) ------- */
/* A batch advances every sample of one or more levels (a mesh and its
 * samples; up to 4 levels, e.g. a multilevel hierarchy) together, one CUDA
 * graph per time step.  Members are FP32 ([component][vertex][sample] with
 * samples innermost); geometry is formed in FP64, the near-equal branch of the
 * log mean runs in FP64, each sample keeps its own FP64 clock and dt (the
 * per-sample time step of src/fv.cc:1499-1618), and ensemble moments are
 * accumulated in FP64.  Euler or Navier-Stokes (constant viscosity law),
 * kepes_tecno_roe / kepes_tecno_rusanov / kepec, first-order or minmod
 * reconstruction, unsteady SSP-RK3, periodic faces and the weak boundary
 * conditions (no strong conditions, no Liou switch).  Boundary values and the
 * viscosity are per sample (tg_batch_set_parameters). */
typedef struct tg_batch tg_batch;
typedef struct tg_batch_level {
  const tg_mesh* mesh;
  const tg_bc_table* bc;       /* boundary kinds; its values start every sample */
  int n_samples;               /* a positive multiple of 32 */
} tg_batch_level;
tg_status tg_batch_create(const tg_batch_level* levels, int n_levels, const tg_material* mat, const tg_options* opt,
                          tg_batch** out);
tg_status tg_batch_destroy(tg_batch* b);
const char* tg_batch_last_error(const tg_batch* b);
/* One sample's state from PrimVar records (caller vertex order); its clock restarts at t = 0. */
tg_status tg_batch_set_state(tg_batch* b, int level, int sample, const double* prim_aos, int n_vertex);
tg_status tg_batch_get_state(tg_batch* b, int level, int sample, double* prim_aos, int n_vertex);
/* Every sample of a level from its random-number row (n_samples x n_rnd, the
 * rnd-file layout of src/fv.cc:502-551), generated on the device: the
 * Kelvin-Helmholtz layer with v' = 0.01 sum_k r_k sin(2 pi k x + 2 pi r_{M+k}),
 * M = n_rnd / 2 (pert type 4, src/perturb.cc:196-208). */
tg_status tg_batch_set_kh(tg_batch* b, int level, const double* rows, int n_rnd);
/* Per-sample uncertain parameters of a level with boundary faces or viscosity
 * (either pointer may be NULL: kept): mu_ref[s] the constant viscosity of
 * sample s, bface_values[(s * n_bface + f) * 10 + q] the tg_bc_table values of
 * reference boundary face f for sample s (e.g. the free stream of a far
 * field).  Kinds stay those of tg_batch_create.  States and clocks are untouched. */
tg_status tg_batch_set_parameters(tg_batch* b, int level, const double* mu_ref, const double* bface_values);
/* Every sample of a level at a uniform state, prim[5 s ..] the PrimVar record
 * (T, p, u, v, w) of sample s (e.g. its free stream); clocks restart at t = 0. */
tg_status tg_batch_set_uniform(tg_batch* b, int level, const double* prim);
/* compute_forces (src/force.cc:116-219) of every sample of a level at its
 * current state, force definitions as for tg_forces:
 * out[(s * n_forces + f) * 4 ..] = inviscid x, y, viscous x, y. */
tg_status tg_batch_forces(tg_batch* b, int level, int n_forces, const int* n_tags, const int* tags, double* out);
/* Steps until every sample has reached output time `instance` (samples that
 * arrive first hold), the run is over, or max_steps steps were issued.
 * info4 (may be NULL): steps issued, min and max elapsed time, samples flagged bad. */
tg_status tg_batch_advance(tg_batch* b, int instance, long max_steps, double* info4);
/* Per-sample elapsed time, output counter and bad flag (any may be NULL). */
tg_status tg_batch_clock(tg_batch* b, int level, double* elapsed, int* counter, int* bad);
/* FP64 ensemble moments of a level's current states, the per-group recurrence of
 * increment_moments applied in sample order (mean by Welford, m2 the sum of
 * squared deviations, sm a Kahan-compensated sum of squares).  Records as for
 * tg_moments_get, extras bits 1 density, 2 mach, 4 entropy. */
tg_status tg_batch_moments(tg_batch* b, int level, int extras, double* fm, double* sm, double* m2);
/* Per-sample FP64 integrals of a level's current states, out[3 s + q]:
 * q0 = sum 0.5 rho v^2 A, q1 = sum 0.5 rho u^2 A, q2 = sum -rho s/(gamma-1) A
 * (the compute_global quantities, src/fv.cc:2186-2203, with the vertical
 * kinetic energy first), periodic copies weighted as there. */
tg_status tg_batch_integrals(tg_batch* b, int level, double* out);
/* Launch shape of the flux and gradient kernels (sample tile x block size,
 * enumerated by TG_BQ_N_SHAPES), and the autotuner that times every shape for
 * `steps` steps from the current state (restored afterwards) and keeps the
 * fastest; ms_out (may be NULL) gets one time per shape. */
tg_status tg_batch_set_shape(tg_batch* b, int shape);
tg_status tg_batch_tune(tg_batch* b, int steps, int* shape_out, double* ms_out);
/* Device time per step over `steps` steps (the batch advances).  A measurement
 * hook with no counterpart in the reference, like tg_time_phase. */
tg_status tg_batch_time_steps(tg_batch* b, int steps, double* ms_per_step);
tg_status tg_batch_stream(tg_batch* b, void** stream_out);
typedef enum {
  TG_BQ_N_LEVELS = 0,
  TG_BQ_KERNELS_PER_STEP = 1,
  TG_BQ_DEVICE_BYTES = 2,
  TG_BQ_SHAPE = 3,
  TG_BQ_SAMPLE_TILE = 4,
  TG_BQ_BLOCK = 5,
  TG_BQ_N_SHAPES = 6
} tg_batch_query_key;
tg_status tg_batch_query(tg_batch* b, int key, double* out);

/* ---- parameter-file expressions evaluated on the device (no counterpart in
 *      the reference, which evaluates its fparser expressions on the host, per
 *      vertex: src/ic.h:79-104, src/bc.h:568-654) ----------------------------- */
/* An expression in the parameter file's syntax (fparser: + - * / % ^, unary -
 * and !, comparisons with fparser's 1e-12 tolerance, & |, the real functions,
 * if(c, a, b)) of x, y, t with pi, the named constants given here (the
 * constants section) and pert(type, x, y, p) (src/perturb.cc:16-208), compiled
 * once on the host.  tg_expr_eval evaluates it on the host for one point and
 * one sample's random numbers (the rnd-file row, src/fv.cc:502-551). */
typedef struct tg_expr tg_expr;
tg_status tg_expr_create(const char* text, int n_const, const char* const* names, const double* values,
                         tg_expr** out);
tg_status tg_expr_destroy(tg_expr* e);
const char* tg_expr_last_error(void);
tg_status tg_expr_eval(const tg_expr* e, double x, double y, double t, const double* rnd, int n_rnd, double* out);
/* InitialCondition::value on the device: fields[0..4] give temperature,
 * x/y/z velocity and pressure (a NULL z velocity is 0); the state of every
 * vertex is evaluated at t = 0 with the random numbers rnd[0 .. n_rnd) and
 * then taken in as tg_set_state takes a state (checked, clocks at t0). */
tg_status tg_set_state_expr(tg_handle* h, const tg_expr* const* fields, const double* rnd, int n_rnd, double t0);
/* The same for every sample of a level, sample s with random numbers
 * rnd_rows[s * n_rnd ..]; clocks restart at t = 0.  A sample whose state has
 * T <= 0 or p <= 0 somewhere makes the call fail (TG_INVALID_ARG) and leaves
 * the level's states undefined until they are set again. */
tg_status tg_batch_set_state_expr(tg_batch* b, int level, const tg_expr* const* fields, const double* rnd_rows,
                                  int n_rnd);
/* Per-sample boundary values of the faces with boundary tag `tag`
 * (BoundaryCondition expressions evaluated at each face vertex at time t):
 * fields as above, a NULL entry keeps that variable's current values. */
tg_status tg_batch_set_bc_expr(tg_batch* b, int level, int tag, const tg_expr* const* fields, const double* rnd_rows,
                               int n_rnd, double t);

/* ---- surrogate network (no counterpart in the reference) ---------------- */
/* The multilayer perceptron din -> 64 -> 64 -> 64 -> dout (GELU) used as the
 * control variate of the multi-fidelity Monte Carlo estimator: FP32 training
 * by hand-written forward / backward passes (mean squared error, Adam, batch
 * reductions in fixed order) and BF16 tensor-core evaluation.  Parameters are
 * one FP32 vector W1[64][din] b1 W2[64][64] b2 W3[64][64] b3 W4[dout][64] b4.
 * din <= 32, dout <= 8. */
typedef struct tg_mlp tg_mlp;
tg_status tg_mlp_create(int din, int dout, unsigned long long seed, tg_mlp** out);
tg_status tg_mlp_destroy(tg_mlp* m);
const char* tg_mlp_last_error(const tg_mlp* m);
int tg_mlp_n_params(const tg_mlp* m);
tg_status tg_mlp_get_params(tg_mlp* m, float* theta);
tg_status tg_mlp_set_params(tg_mlp* m, const float* theta);    /* also resets the optimiser */
/* Mean squared error of one batch and its gradient with respect to theta. */
tg_status tg_mlp_loss_grad(tg_mlp* m, const float* X, const float* T, int n, float* loss, float* grad);
/* Adam over `epochs` passes of in-order mini-batches; losses[epoch] = last batch loss. */
tg_status tg_mlp_train(tg_mlp* m, const float* X, const float* T, int n, int epochs, int batch, float lr,
                       float* losses);
/* precision 0: FP32, 1: BF16 tensor cores; on_device: X and Y are device pointers. */
tg_status tg_mlp_predict(tg_mlp* m, const float* X, int n, float* Y, int precision, int on_device);

/* ---- allocation-free residual norm ------------------------------------ */

#define TG_NOALLOC_MAX_VERTICES 268435456

/* No counterpart in the reference (whose norm is a member of FiniteVolume
 * working on its own arrays).  For callers that cannot allocate device memory
 * while they run -- hosts that reserve all GPU memory up front, code running
 * while another part of the program captures a CUDA graph, real-time loops --
 * this computes the residual norms of compute_residual_norm
 * (src/fv.cc:1801-1879) from buffers the caller already owns, with no handle
 * and no cudaMalloc/cudaFree: its scratch is a fixed 64 KiB device array in
 * the library, held by every GPU that loads it until exit.
 *   res_dev     device array n_vertex x 5, the reference's Flux layout
 *               (mass, mx, my, mz, energy); the z component is ignored.  With
 *               strong boundary conditions the caller passes the residual
 *               with the no-slip momentum already zeroed, as
 *               compute_residual_norm zeroes it first (src/fv.cc:1807-1819)
 *               and as tg_residual returns it; the entry point sums what it
 *               is given
 *   dcarea_dev  device array n_vertex, dual areas
 *   weight_dev  device array n_vertex, 1/|P_i| for periodic vertices, else 1
 *   total0      normaliser; <= 0 marks the first iteration (total becomes it)
 *   out6_dev    device array of 6: mass, mx, my, energy norms, normalised
 *               total, normaliser
 *   stream      cudaStream_t (NULL = default stream); the call is
 *               asynchronous on it.
 * n_vertex must be at most TG_NOALLOC_MAX_VERTICES (TG_INVALID_ARG otherwise).
 * The norms are those of one whole mesh: each component is divided by
 * n_vertex, so the entry point serves single-partition meshes.  (The
 * reference's partitioned norm weights shared vertices by 1/nbs and divides by
 * the global vertex count, src/fv.cc:1830-1859; per-partition calls do not
 * give it.)
 * The first call on each device looks up the scratch array's device address,
 * so make it before any stream capture that should contain later calls.  The
 * address is kept for the life of the process: do not call the entry point
 * on a device after cudaDeviceReset on it.
 * All calls share the scratch array: calls whose kernels overlap on the GPU
 * (e.g. on two streams) race and may return wrong norms.
 * On failure tg_noalloc_last_error() describes the problem. */
tg_status tg_residual_norm_noalloc(const double* res_dev, const double* dcarea_dev, const double* weight_dev,
                                   int n_vertex, double total0, double* out6_dev, void* stream);
const char* tg_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* TENSUM_GPU_H */
